/* C ABI of the B200-native exact volumetric ellipsoid tracer (libever_b200.so).
 *
 * Drop-in replacement for the native layer under EVER's Python API
 * splinetracers/fast_ellipsoid_splinetracer.py:222-256 (trace_rays). In the
 * reference that layer is a pybind11 module (splinetracers/fast_ellipsoid_splinetracer/
 * py_binding.cpp:261-282) over OptiX plus two slangtorch kernels; here it is plain C:
 * device pointers and sizes in, status code out, message via ever_last_error().
 *
 * Conventions
 *  - All float/int pointers are DEVICE pointers (CUDA global memory) unless noted.
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream.
 *  - No function allocates device memory, synchronises the host, or throws: callers
 *    pass workspaces sized by the *_workspace_bytes() functions, and every call only
 *    enqueues kernels on `stream`, so the calls can be captured in a CUDA graph.
 *  - Return value: EVER_OK (0) or an EVER_ERR_* code; ever_last_error() then holds a
 *    message (thread-local).
 *  - Ellipsoid parameters follow the reference: mean (N,3), scale (N,3), quat (N,4)
 *    as (r,x,y,z) and not required to be unit, density (N), features (N,K,3) SH
 *    coefficients, all fp32 contiguous.
 */
#ifndef EVER_B200_H
#define EVER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EVER_OK 0
#define EVER_ERR_INVALID 1   /* bad argument (shape, null pointer, size) */
#define EVER_ERR_CUDA 2      /* a CUDA launch or API call failed */
#define EVER_ERR_WORKSPACE 3 /* workspace too small */

#define EVER_ABI_VERSION 2

/* A scene built by ever_scene_build(): a binary LBVH over the ellipsoids plus their
 * intersection records, both in Morton order, all inside the caller's workspace.
 * Replaces the reference's Primitives + GAS objects (py_binding.cpp:94-149,
 * GAS.cpp:56-154, create_aabbs.cu:69-132). Plain data: may be copied by value. */
typedef struct EverScene {
  int64_t num_prims;  /* N */
  int32_t sh_coeffs;  /* K: SH coefficients stored per ellipsoid (feature stride) */
  int32_t num_nodes;  /* internal BVH nodes: max(N-1, 1), 0 if N == 0 */
  void* nodes;        /* num_nodes x 64 B: child boxes + child links */
  void* records;      /* N x 64 B: 3x3 local-frame matrix, mean, density, DC colour */
  float* features;    /* N rows of 3K floats padded to a multiple of 4, Morton order */
  int32_t* order;     /* N: Morton position -> original ellipsoid index */
  void* scratch;      /* build-time scratch inside the workspace */
} EverScene;

/* Launch configuration chosen by the autotuner (0 = built-in default). */
typedef struct EverTune {
  int32_t kbuf;       /* events gathered per traversal round: 8, 16 or 32 */
  int32_t block;      /* threads per block: 64, 128 or 256 */
  int32_t traversal;  /* 0 (default): warp packets, each first taking the leaves its rays can meet in
                         one breadth-first walk and integrating them in order (the frustum phase),
                         then gather rounds for any ray it could not finish; 1: one walk per ray;
                         2: warp packets, gather rounds only */
  int32_t regroup_min;/* ever_trace_forward_regrouped: a pass with fewer rays than this runs every
                         remaining round instead of handing the rest on; 0: four times the GPU's
                         resident lanes */
  int32_t stack_depth;/* traversal stack entries in use, 8..64 (0: 64); a tree deeper than the stack
                         raises EVER_STATUS_STACK_OVERFLOW (a subtree is skipped) */
  int32_t reserved[3];
} EverTune;

/* Per-ray outputs of a forward trace. Null pointers are skipped unless noted. */
typedef struct EverForwardOut {
  float* out;          /* (R,5) RGB, opacity, distortion (required) */
  float* states;       /* (R,16) final SplineState (structs.h:41-53 layout); needed by backward */
  float* last_dirac;   /* (R,4) dirac of the last consumed event */
  int32_t* iters;      /* (R) consumed events (required) */
  int32_t* event_log;  /* (slots, log_cap) ray-major event ids in Morton numbering
                          (2j+1 entry, 2j exit): row = launch slot (ray ray_order[slot], or
                          ray slot without ray_order), entries in event order, so a ray's
                          replay reads consecutive words; needed by backward.
                          ever_event_log_to_reference gives the reference's layout */
  int32_t log_cap;     /* entries per row of event_log (>= max_iters to log every event) */
  int32_t* touch_count;/* (N) original order: events per ellipsoid (atomic, exact) */
  float* ray_stats;    /* (R,2): consumed events, termination depth (t of last event) */
  int32_t* status;     /* (1) OR of EVER_STATUS_* flags raised by the kernels */
} EverForwardOut;

#define EVER_STATUS_STACK_OVERFLOW 1
#define EVER_STATUS_LOG_OVERFLOW 2
#define EVER_STATUS_INIT_OVERFLOW 4

/* Gradients of a backward trace. Prim gradients are written in original order and
 * clipped as fast_ellipsoid_splinetracer.py:204-219 clips them. */
typedef struct EverBackwardOut {
  float* dmean;      /* (N,3) */
  float* dscale;     /* (N,3) */
  float* dquat;      /* (N,4) */
  float* ddensity;   /* (N) */
  float* dfeatures;  /* (N,K,3) */
  float* drayo;      /* (R,3) */
  float* drayd;      /* (R,3) */
  float* dmeans2d;   /* (N,2) or NULL; needs wct */
} EverBackwardOut;

typedef struct EverTraceArgs {
  float tmin;
  float tmax;
  int32_t max_iters;
  int32_t sh_degree;  /* colour of an event. -1 (default): the reference's forward colour,
                         the ellipsoid's DC term C0*f0 + 0.5 whatever K (shaders.slang:72-75,
                         eval_sh_col0), and its gradient in the backward (features k >= 1 get
                         zero); 0..3: SH of that degree along the raw rayd in both passes */
  const float* depth_hint; /* (R) device, nullable: a guess per ray of the t at which it stops (e.g.
                              the ray-cost model's). A packet's first frustum stage then covers the
                              t range up to its largest guess instead of the whole scene; rays that
                              go on continue in the next stage. Results do not depend on it. */
} EverTraceArgs;

const char* ever_last_error(void);
int ever_abi_version(void);

/* Bytes of workspace ever_scene_build() needs for N ellipsoids with K SH coefficients. */
size_t ever_scene_workspace_bytes(int64_t num_prims, int32_t sh_coeffs);

/* Builds the scene: AABBs of the ellipsoids (create_aabbs.cu:69-115), 30-bit Morton
 * codes, an on-device LSD radix sort, a Karras LBVH and a bottom-up box refit; then
 * reorders records and features into Morton order. Replaces Primitives.add_primitives
 * + GAS (py_binding.cpp:99-132, GAS.cpp:56-154). */
int ever_scene_build(const float* mean, const float* scale, const float* quat, const float* density,
                     const float* features, int64_t num_prims, int32_t sh_coeffs, void* workspace,
                     size_t workspace_bytes, EverScene* scene, void* stream);

/* ever_scene_build for traces that use the DC colour only (sh_degree 0 / the default, the
 * reference forward's colour): every record gets its DC colour C0 * f0 + 0.5 from
 * `features`, but the feature rows are not copied into the workspace (scene->features is
 * NULL). A trace with sh_degree > 0 on such a scene fails with EVER_ERR_INVALID;
 * ever_scene_set_features and ever_scene_refit update the DC colours. Same workspace as
 * ever_scene_build. No counterpart in the reference (its GAS build copies every
 * feature); trace_rays uses it at its default colour. */
int ever_scene_build_dc(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* features, int64_t num_prims, int32_t sh_coeffs, void* workspace,
                        size_t workspace_bytes, EverScene* scene, void* stream);

/* Replaces the features of a built scene (same N and K) without rebuilding the BVH.
 * Counterpart of Primitives.set_features + Forward.update_model (py_binding.cpp:133-138, 207-209). */
int ever_scene_set_features(EverScene* scene, const float* features, void* stream);

/* Refits a scene built by ever_scene_build on the same workspace to new ellipsoid
 * parameters (same N and K): records, boxes and (when features is not NULL) features are
 * recomputed, the tree keeps the last build's Morton order and topology and is refitted
 * bottom-up. Much cheaper than a rebuild between small parameter updates (training steps);
 * traversal gets slower as ellipsoids move far from where they were built. No counterpart
 * in the reference, which rebuilds its GAS on every call (GAS.cpp:56-154). */
int ever_scene_refit(const float* mean, const float* scale, const float* quat, const float* density,
                     const float* features, void* workspace, size_t workspace_bytes, EverScene* scene, void* stream);

/* Forward trace of R rays: rayo/rayd (R,3). Counterpart of Forward.trace_rays
 * (py_binding.cpp:210-258, Forward.cpp:23-82, shaders.slang:171-235), including the
 * initial density of rays that start inside ellipsoids (initialize_density.cu:152-208).
 * ray_order (R, nullable): the order in which threads pick rays up (a permutation);
 * results are written by ray index and do not depend on it. */
int ever_trace_forward(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                       const EverTraceArgs* args, const int32_t* ray_order, const EverTune* tune,
                       const EverForwardOut* out, void* stream);

/* Bytes of workspace ever_trace_forward_regrouped() needs for R rays (0 if R is out of
 * range). */
size_t ever_trace_forward_workspace_bytes(int64_t num_rays);

/* ever_trace_forward, same arguments and the same results bit for bit, for warp-packet
 * traversal (tune->traversal is ignored), and faster: after each of the first two gather
 * rounds the rays that need more rounds are packed into full warps in launch order, so
 * warps stop running with most of their lanes idle. Rays between passes keep their loop
 * state in out->states and out->last_dirac, which are therefore required. R < 2^31.
 * No counterpart in the reference (OptiX runs one thread per ray to the end). */
int ever_trace_forward_regrouped(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                                 const EverTraceArgs* args, const int32_t* ray_order, const EverTune* tune,
                                 const EverForwardOut* out, void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of gradient-accumulation workspace ever_trace_backward() needs. */
size_t ever_backward_workspace_bytes(int64_t num_prims, int32_t sh_coeffs);

/* Backward of a forward trace: grad_out (R,5); states/iters/event_log from the forward.
 * Counterpart of SplineTracer.backward (fast_ellipsoid_splinetracer.py:106-219) with
 * backwards_kernel and backwards_initial_drgb_kernel (backwards_kernel.slang:259-428).
 * wct (4x4 row-major, nullable) with num_wct matrices: ray r uses wct[r] if r < num_wct,
 * else wct[0], for dmeans2d as backwards_kernel.slang:313-321. */
int ever_trace_backward(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                        const EverTraceArgs* args, const float* grad_out, const float* states,
                        const int32_t* iters, const int32_t* event_log, int32_t log_cap,
                        const float* wct, int32_t num_wct, const float* mean, const float* scale,
                        const float* quat, void* workspace, size_t workspace_bytes,
                        const int32_t* ray_order, const EverTune* tune, const EverBackwardOut* out,
                        void* stream);

/* ever_trace_backward with its own launch order: launch position p replays forward slot
 * slot_order[p] (a permutation of 0..R-1; the event-log column), ray ray_order[slot].
 * The results do not depend on the order (up to the summation order of the
 * ellipsoid gradients). No counterpart in the reference. */
int ever_trace_backward_ordered(const EverScene* scene, const float* rayo, const float* rayd, int64_t num_rays,
                                const EverTraceArgs* args, const float* grad_out, const float* states,
                                const int32_t* iters, const int32_t* event_log, int32_t log_cap, const float* wct,
                                int32_t num_wct, const float* mean, const float* scale, const float* quat,
                                void* workspace, size_t workspace_bytes, const int32_t* ray_order,
                                const int32_t* slot_order, const EverTune* tune, const EverBackwardOut* out,
                                void* stream);

/* A backward launch order from the forward's per-ray event counts (iters, indexed by
 * ray; ray_order: the forward's order, nullable): slots whose rays consumed more events
 * come first, grouped by min(iters >> shift, 255), the forward's coherent slot order
 * inside a group. Warps then replay rays of equal length. Same workspace as
 * ever_ray_order. No counterpart in the reference. */
int ever_backward_slot_order(const int32_t* iters, const int32_t* ray_order, int64_t num_rays, int32_t shift,
                             void* workspace, size_t workspace_bytes, int32_t* slot_order, void* stream);

/* Converts an event log in Morton numbering into the reference's tri_collection ids
 * (2p+1 entry, 2p exit with original indices p; fast_ellipsoid_splinetracer.py:93-101),
 * (max_iters, R) indexed by ray. ray_order: the order the forward was launched with.
 * Entries at or beyond iters[r] are set to 0, as the reference's zero-filled buffer. */
int ever_event_log_to_reference(const EverScene* scene, const int32_t* event_log, int32_t log_cap,
                                const int32_t* iters, int64_t num_rays, const int32_t* ray_order,
                                int32_t* tri_collection, int32_t max_iters, void* stream);

/* Bytes of workspace ever_ray_order() needs for R rays. */
size_t ever_ray_order_workspace_bytes(int64_t num_rays);

/* A coherent launch order for R rays (no counterpart in the reference, whose OptiX
 * launch order is the ray index): rays sorted by a coarse origin cell and the Hilbert
 * index of their octahedral direction, so each warp's packet covers a compact patch.
 * Writes a permutation of 0..R-1 to ray_order (R). Pass it to forward and backward. */
int ever_ray_order(const float* rayo, const float* rayd, int64_t num_rays, void* workspace,
                   size_t workspace_bytes, int32_t* ray_order, void* stream);

/* ever_ray_order for callers that cannot allocate device memory: no workspace argument
 * and no allocation inside. No counterpart in the reference. Meant for callers such as a
 * viewer's or render server's frame loop that must never block on the allocator (cudaFree
 * waits for the whole device), or a binding from another runtime that cannot hand this
 * library a workspace. Its scratch is a static device array of about 33 MB built into the
 * library, held by every GPU that loads it until exit; num_rays must be <= 2,097,152 (one
 * 1920x1080 view), larger counts return EVER_ERR_INVALID. Each call outside a stream
 * capture looks the array's address up (cudaGetSymbolAddress) and keeps it for calls made
 * during a capture, so make one call on a device before capturing there; calls that
 * overlap on the GPU share the array and race, so order them (e.g. one stream). Same
 * output as ever_ray_order. */
int ever_ray_order_static(const float* rayo, const float* rayd, int64_t num_rays, int32_t* ray_order,
                          void* stream);

/* ---- batched persistent tracing (many views over several scenes per launch) ----
 * No counterpart in the reference, which launches OptiX once per view. A batch lists
 * views (a range of rays traced against one built scene). Each view's rays get their own
 * coherent order and are padded to whole 32-ray packets, so a warp's packet never mixes
 * scenes; persistent warps take packets from a device counter in packet order. */
typedef struct EverBatchView {
  int32_t scene;      /* index into the scenes array given to ever_batch_setup */
  int32_t pad;
  int64_t ray_offset; /* first ray of the view in the concatenated ray arrays */
  int64_t ray_count;
} EverBatchView;

typedef struct EverBatch {  /* filled by ever_batch_setup; plain data */
  int32_t num_scenes;
  int32_t num_views;
  int64_t num_slots;  /* padded packet slots: event-log columns of a batched forward */
  int64_t num_rays;
  void* scene_table;  /* device: one row per scene (pointers into the built scenes) */
  void* view_table;   /* device: one row per view */
  int32_t* slot_ray;  /* device (num_slots): ray index per slot, -1 for padding */
  uint32_t* counters; /* device: work counters of the persistent launches */
  void* order_scratch;/* device: ray-order sort scratch */
  int32_t sh_coeffs[64]; /* host copy: K of each scene */
  int64_t num_prims[64]; /* host copy: N of each scene */
  void* bwd_workspace[64];/* host copy: backward workspace of each scene (or NULL) */
} EverBatch;

/* Bytes of batch workspace for these views (host array); *num_slots receives the padded
 * slot count. At most 64 views and 64 scenes; the views must tile the concatenated rays
 * in order (view v starts where view v-1 ends, the first at ray 0). */
size_t ever_batch_workspace_bytes(int32_t num_scenes, const EverBatchView* views, int32_t num_views,
                                  int64_t* num_slots);

/* Lays the batch out in `workspace` and uploads the scene and view tables. scenes: host
 * array of built scenes; bwd_workspaces: host array of per-scene backward workspaces
 * (ever_backward_workspace_bytes each; entries may be NULL for forward-only use). This
 * set-up call copies the tables synchronously; later calls only enqueue work. */
int ever_batch_setup(const EverScene* scenes, void* const* bwd_workspaces, int32_t num_scenes,
                     const EverBatchView* views, int32_t num_views, int64_t num_rays, void* workspace,
                     size_t workspace_bytes, EverBatch* batch);

/* Coherent order inside every view (ever_ray_order per view), written to the slot map. */
int ever_batch_order(const EverBatch* batch, const float* rayo, const float* rayd, void* stream);

/* One persistent forward launch over all views. Outputs are indexed by ray; event_log
 * has batch->num_slots rows of log_cap entries. The colour follows args->sh_degree as in
 * ever_trace_forward; every scene must hold the coefficients it needs. */
int ever_trace_forward_batched(const EverBatch* batch, const float* rayo, const float* rayd,
                               const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                               void* stream);

/* One persistent backward launch over all views: accumulates every scene's gradients into
 * its backward workspace (zeroed here) and writes the ray gradients (clipped). */
int ever_trace_backward_batched(const EverBatch* batch, const float* rayo, const float* rayd,
                                const EverTraceArgs* args, const float* grad_out, const float* states,
                                const int32_t* iters, const int32_t* event_log, int32_t log_cap, float* drayo,
                                float* drayd, const EverTune* tune, void* stream);

/* Turns one scene's accumulated gradients (its backward workspace) into dmean, dscale,
 * dquat, ddensity, dfeatures (clipped as fast_ellipsoid_splinetracer.py:204-219). The
 * workspace's last num_prims int32 are scratch (the inverse Morton order). */
int ever_scene_finalize_gradients(const EverScene* scene, const float* mean, const float* scale,
                                  const float* quat, void* bwd_workspace, size_t bwd_workspace_bytes,
                                  const EverBackwardOut* out, void* stream);

/* ---- learned ray-cost model and cost-binned ray orders ----
 * No counterpart in the reference. A 39 -> 64 -> 64 -> 2 ReLU MLP predicts each ray's
 * cost [log(1 + consumed events), depth offset / scale] from a sinusoidal encoding of the
 * point of the ray's line closest to the scene centre (x, sin(2^k pi x), cos(2^k pi x),
 * k = 0..5). BF16 weights and activations, FP32 accumulation, tcgen05 tensor cores. It is
 * trained on the tracer's own per-ray logs (EverForwardOut.ray_stats) and its predicted
 * cost bins order rays: costlier bins first, each in the coherent order. Results of the
 * trace do not depend on the order. */
#define EVER_MLP_PARAMS 9360
typedef struct EverMlp {
  float* params;    /* device fp32 [EVER_MLP_PARAMS]: W1 [64x64], W2 [64x64], W3 [16x64] (row =
                       output unit), b1 [64], b2 [64], b3 [16]; W1 columns 39..63 and W3 rows
                       2..15 are padding and must stay zero */
  void* w1;         /* device bf16 copies of W1, W2, W3 read by the tensor cores; refreshed */
  void* w2;         /* by ever_mlp_pack and ever_mlp_adam */
  void* w3;
  float centre[3];  /* scene centre of the encoding */
  float inv_scale;  /* 1 / scene scale of the encoding */
  int64_t wait_clocks; /* bound in clocks of each wait for the tensor cores (0: 2^31, about a
                          second); a wait that runs out sets *error, lets the MMAs in flight
                          finish and frees the tensor memory. Tests set a few clocks. */
} EverMlp;

/* Bytes of workspace ever_mlp_gradients needs (per-CTA partial gradients). */
size_t ever_mlp_workspace_bytes(void);

/* Rounds the fp32 weights to the bf16 copies. */
int ever_mlp_pack(const EverMlp* mlp, void* stream);

/* Predictions pred (num_rays, 2) for rays (rayo, rayd) or for pre-encoded inputs feat
 * (num_rays, 64; used when not NULL). bins (nullable): cost bin of each ray, the number of
 * thresholds[0..2] (host array) that pred[., 0] exceeds. error: device int32 set to 1 if a
 * tensor-core wait timed out (the outputs are then invalid). */
int ever_mlp_predict(const EverMlp* mlp, const float* rayo, const float* rayd, const float* feat, int64_t num_rays,
                     float* pred, uint8_t* bins, const float* thresholds, int32_t* error, void* stream);

/* Gradient of the weighted squared error mean_s(w0 (y0 - t0)^2 + w1 (y1 - t1)^2) over the
 * samples s (ray sample_idx[s], or s when sample_idx is NULL; target (rays, 2)) with respect
 * to the fp32 parameters, written to grads [EVER_MLP_PARAMS]; the loss to *loss (nullable).
 * Deterministic for a given device. */
int ever_mlp_gradients(const EverMlp* mlp, const float* rayo, const float* rayd, const float* feat,
                       const int32_t* sample_idx, int64_t num_samples, const float* target, float loss_w0,
                       float loss_w1, float* grads, float* loss, void* workspace, size_t workspace_bytes,
                       int32_t* error, void* stream);

/* One Adam step (step counts from 1) on the fp32 parameters; refreshes the bf16 copies. */
int ever_mlp_adam(const EverMlp* mlp, const float* grads, float* adam_m, float* adam_v, float lr, float beta1,
                  float beta2, float eps, int32_t step, void* stream);

/* ever_ray_order with cost bins (one byte per ray, 0..3, larger = costlier) on top of the
 * key: costlier bins come first. Same workspace as ever_ray_order. */
int ever_ray_order_binned(const float* rayo, const float* rayd, const uint8_t* bins, int64_t num_rays,
                          void* workspace, size_t workspace_bytes, int32_t* ray_order, void* stream);

/* ever_batch_order with cost bins: inside every view, costlier bins first. */
int ever_batch_order_binned(const EverBatch* batch, const float* rayo, const float* rayd, const uint8_t* bins,
                            void* stream);

/* ---- trained scenes from binary PLY files (host code) ----
 * The reference's scene file layout and conversion (ply_file_loader.cc:166-293): per vertex
 * 62 little-endian floats (mean, normal, 48 SH values, opacity, scale, rotation), turned
 * into means, quaternions q/(q.q), scales min(softplus(s)+3e-4, 25), densities
 * -log(1 - 0.99 sigmoid(opacity)) / (2 min scale) and SH features (N,16,3). */

/* Number of ellipsoids in the file, or -1 (see ever_last_error) if it is not a valid file. */
int64_t ever_ply_count(const char* path);

/* Reads the file into HOST buffers of `capacity` ellipsoids: mean (N,3), scale (N,3),
 * quat (N,4), density (N), features (N,16,3). */
int ever_ply_read(const char* path, int64_t capacity, float* mean, float* scale, float* quat, float* density,
                  float* features);

/* ---- the trainer's per-ellipsoid colour pre-pass and camera ray generation ---- */

/* Colour of each ellipsoid seen from the camera centre cam_pos (device, 3 floats): SH of
 * degree sh_degree (features (N,K,3), K >= (sh_degree+1)^2) in the direction
 * normalize(mean - cam_pos), plus 0.5. Counterpart of eval_sh.EvalSH.forward / sh_kernel
 * (eval_sh.py:28-56, sh_kernel.slang:21-43). mode 0 writes that colour (N,3); mode 1 writes
 * the trainer's tracer features RGB2SH(softplus(colour, beta=10)) (N,1,3) in the same pass
 * (integration_utils/gaussian_renderer/ever.py:178-180). */
int ever_sh_prepass(const float* mean, const float* features, int64_t num_prims, int32_t sh_coeffs,
                    int32_t sh_degree, const float* cam_pos, int32_t mode, float* out, void* stream);

/* Gradient of ever_sh_prepass with respect to the features, written in full to
 * grad_features (N,K,3) (entries of degree > sh_degree are zero). Counterpart of
 * EvalSH.backward / bw_sh_kernel (eval_sh.py:58-69, sh_kernel.slang:45-99), including its
 * skip of ellipsoids whose colour gradient is below 1e-8 in every channel. */
int ever_sh_prepass_backward(const float* mean, const float* features, int64_t num_prims, int32_t sh_coeffs,
                             int32_t sh_degree, const float* cam_pos, int32_t mode, const float* grad_out,
                             float* grad_features, void* stream);

typedef struct EverCamera {
  int32_t width, height;
  float fx, fy;     /* focal lengths in pixels */
  float cx, cy;     /* principal point in pixels (the reference uses width/2, height/2) */
  float c2w[12];    /* camera-to-world 3x4, row-major: rayd = c2w[:, :3] d, rayo = c2w[:, 3] */
} EverCamera;

/* One ray per pixel, row-major: d = normalize(((col + ox) - cx) / fx, ((row + oy) - cy) / fy, 1),
 * rayd = R d, rayo = camera centre. jitter (nullable, device (width*height, 2)) gives the
 * per-pixel offsets (ox, oy); NULL means pixel centres (0.5, 0.5). Counterpart of
 * camera2rays / get_ray_directions / get_rays (integration_utils/gaussian_renderer/ever.py:29-74,105-118). */
int ever_camera_rays(const EverCamera* camera, const float* jitter, float* rayo, float* rayd, void* stream);

/* ---- camera traces: the trace makes each pixel's ray from the camera itself ----
 * The counterpart of camera2rays followed by trace_rays (integration_utils/gaussian_renderer/
 * ever.py:105-121, 189-205) without the (R,6) ray arrays: the rays are those of
 * ever_camera_rays (same arithmetic, bit for bit). Threads take "slots", 32 per 8x4 pixel
 * tile, so that a warp traces one tile. Tiles are grouped in 64x64-pixel supertiles
 * (8 x 16 tiles), supertiles row-major, tiles inside a supertile in Morton order: slot s
 * lies in supertile u = s / 4096 at (u % ceil(width/64), u / ceil(width/64)), in its tile
 * w = (s / 32) % 128 at (tx, ty) = bits (0,2,4) and (1,3,5,6) of w, and is pixel
 * (col, row) = (64 ux + 8 tx + s % 8, 64 uy + 4 ty + (s % 32) / 8), or padding (no pixel)
 * where that lies outside the image. Per-pixel outputs are indexed by pixel (row-major,
 * R = width*height); event-log columns are slots (row length ever_camera_slots). */

/* Slot count ceil(width/64) * ceil(height/64) * 4096, or -1 (see ever_last_error). */
int64_t ever_camera_slots(const EverCamera* camera);

/* slot_pixel (slots): the pixel of each slot, -1 for padding. */
int ever_camera_slot_pixels(const EverCamera* camera, int32_t* slot_pixel, void* stream);

/* Forward trace of the camera's rays; as ever_trace_forward otherwise (tune->traversal is
 * ignored: warps always trace their tile as one packet). */
int ever_trace_forward_camera(const EverScene* scene, const EverCamera* camera, const float* jitter,
                              const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                              void* stream);

/* ever_trace_forward_camera with the passes of ever_trace_forward_regrouped (the same
 * results bit for bit): out->states and out->last_dirac are required, and the workspace
 * holds ever_trace_forward_workspace_bytes(ever_camera_slots(camera)) bytes. No counterpart
 * in the reference. */
int ever_trace_forward_camera_regrouped(const EverScene* scene, const EverCamera* camera, const float* jitter,
                                        const EverTraceArgs* args, const EverTune* tune, const EverForwardOut* out,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* Backward of ever_trace_forward_camera; as ever_trace_backward otherwise. slot_order
 * (nullable): launch position -> slot, from ever_camera_backward_slot_order. out->drayo and
 * out->drayd may both be NULL (camera rays need no gradient); else (R,3) by pixel. */
int ever_trace_backward_camera(const EverScene* scene, const EverCamera* camera, const float* jitter,
                               const EverTraceArgs* args, const float* grad_out, const float* states,
                               const int32_t* iters, const int32_t* event_log, int32_t log_cap, const float* wct,
                               int32_t num_wct, const float* mean, const float* scale, const float* quat,
                               void* workspace, size_t workspace_bytes, const int32_t* slot_order,
                               const EverTune* tune, const EverBackwardOut* out, void* stream);

/* ever_backward_slot_order for a camera trace (iters by pixel; padding slots last).
 * Workspace: ever_ray_order_workspace_bytes(ever_camera_slots(camera)). */
int ever_camera_backward_slot_order(const EverCamera* camera, const int32_t* iters, int32_t shift, void* workspace,
                                    size_t workspace_bytes, int32_t* slot_order, void* stream);

/* ever_event_log_to_reference for a camera trace: tri_collection (max_iters, R) by pixel. */
int ever_camera_event_log_to_reference(const EverScene* scene, const EverCamera* camera, const int32_t* event_log,
                                       int32_t log_cap, const int32_t* iters, int32_t* tri_collection,
                                       int32_t max_iters, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EVER_B200_H */
