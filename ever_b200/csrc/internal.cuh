// Host-side internals shared by the translation units of libever_b200.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "ever_b200.h"

namespace ever {

// Records a message for ever_last_error() and returns code (defined in capi.cu).
int set_last_error(int code, const char* msg);

// Bump allocator over a caller-provided workspace: 256-byte aligned segments.
struct WsCursor {
  int64_t offset = 0;
  int64_t take(int64_t bytes) {
    const int64_t at = offset;
    offset += (std::max<int64_t>(bytes, 0) + 255) / 256 * 256;
    return at;
  }
};

struct SceneLayout {
  int64_t nodes, records, features, order;
  int64_t aabb_a, aabb_b, keys_a, keys_b, vals_a, vals_b, hist;
  int64_t parent_node, parent_leaf, flags, bounds;
  int nblocks;
  int64_t total;
};

SceneLayout scene_layout(int64_t N, int K);
int sort_blocks(int64_t N);
void sort_pairs(uint32_t*& ka, uint32_t*& va, uint32_t*& kb, uint32_t*& vb, uint32_t* hist, int64_t N, int bits,
                cudaStream_t st);
int64_t ray_order_workspace(int64_t R);
struct BatchView;
// bins (nullable, one byte per ray, 0..3, larger = costlier): when given, rays of a higher
// cost bin come first, each bin in the usual coherent order.
cudaError_t batch_ray_order(const float* rayo, const float* rayd, int64_t R, const BatchView* views, int num_views,
                            char* ws, int32_t* slot_ray, int64_t num_slots, cudaStream_t st,
                            const uint8_t* bins = nullptr);
cudaError_t ray_order(const float* rayo, const float* rayd, int64_t R, char* ws, int32_t* order, cudaStream_t st,
                      const uint8_t* bins = nullptr);
// Backward launch order over forward slots: slots whose rays consumed more events first
// (key min(iters >> shift, 255), descending), the forward's slot order inside a key.
// ray_order[s] < 0 marks a padding slot (sorted last). Workspace: ray_order_workspace(R).
cudaError_t backward_slot_order(const int32_t* iters, const int32_t* ray_order, int64_t R, int shift, char* ws,
                                int32_t* slot_order, cudaStream_t st, const BatchView* views = nullptr,
                                int num_views = 0);
// dc_only: the scene keeps only each record's DC colour, no feature rows (sc->features null).
cudaError_t scene_build(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* feat, int64_t N, int K, char* ws, const SceneLayout& L, EverScene* sc,
                        cudaStream_t st, bool dc_only = false);
cudaError_t scene_set_features(EverScene* sc, const float* feat, cudaStream_t st);
cudaError_t scene_refit(const float* mean, const float* scale, const float* quat, const float* density,
                        const float* feat, char* ws, const SceneLayout& L, EverScene* sc, cudaStream_t st);

struct FwdParams {
  const void* nodes;
  const void* records;
  const float* features;
  const int32_t* order;
  int64_t N;
  int K;
  const float* rayo;
  const float* rayd;
  int64_t R;
  float tmin, tmax;
  int max_iters;
  const int32_t* ray_order;
  EverForwardOut out;
  int frustum;  // packet kernels: frustum phase before the rounds (set from the tune)
  int stack_depth;  // traversal stack entries in use, <= kStackDepth (set from the tune)
  const float* depth_hint;  // (R) nullable: per-ray guess of the stopping t (first frustum stage)
};

cudaError_t launch_forward(const FwdParams& P, int deg, const EverTune& tune, cudaStream_t st);

// Regrouped forward (warp packets): round 0 for every ray, then the rays still active are
// packed into full warps for round 1, and again for the remaining rounds. Scratch in the
// caller's workspace; P.out.states and P.out.last_dirac hold the parked rays' loop state.
struct RegroupScratch {
  uint32_t* mask0;    // ceil(R/32): lanes of each pass-0 warp still active
  uint32_t* mask1;    // ceil(R/32): the same for pass 1
  uint32_t* offsets;  // ceil(R/32) + 1: exclusive scan of a mask's popcounts
  int32_t* list1;     // R: slots of pass 1, in slot order
  int32_t* list2;     // R: slots of pass 2
  uint32_t* count1;   // 1
  uint32_t* count2;   // 1
  int64_t split_min;  // a pass with fewer rays runs every remaining round (set by the launcher)
};
int64_t regroup_workspace(int64_t R);
RegroupScratch regroup_scratch(char* ws, int64_t R);
// dst = the entries of src (identity if null) at the positions whose mask bit is set, in
// order; *dst_count = their number. n: number of positions (*n_dev if given, else n_max).
cudaError_t regroup_compact(const uint32_t* mask, const uint32_t* n_dev, int64_t n_max, const int32_t* src,
                            uint32_t* offsets, int32_t* dst, uint32_t* dst_count, cudaStream_t st);
struct CameraParams;
// cam: null for the ray arrays of P, else the camera whose slots are traced (rays made in
// the kernels, P.R = its pixel count) with the per-pixel jitter (nullable).
cudaError_t launch_forward_regrouped(const FwdParams& P, const RegroupScratch& W, const CameraParams* cam,
                                     const float* jitter, int deg, const EverTune& tune, cudaStream_t st);
template <int KBUF>
cudaError_t launch_forward_regrouped_k(const FwdParams& P, const RegroupScratch& W, const CameraParams* cam,
                                       const float* jitter, int deg, int block, cudaStream_t st);
// Per k-buffer size launchers (trace_fwd_k8.cu, trace_fwd_k16.cu, trace_fwd_k32.cu).
template <int KBUF>
cudaError_t launch_forward_k(const FwdParams& P, int deg, int block, int traversal, cudaStream_t st);

// ---- batched persistent launches: many views over several scenes in one launch ----
struct BatchScene {  // one row of the device-side scene table
  const void* nodes;
  const void* records;
  const float* features;
  const int32_t* order;
  int64_t N;
  int32_t K;
  int32_t pad;
  float* acc_geo;   // backward accumulators of this scene (Morton order)
  float* acc_feat;
};

struct BatchView {  // slots [slot_offset, slot_offset + slot_count) belong to one scene
  int64_t slot_offset;  // a multiple of 32: a warp's packet never mixes views
  int64_t slot_count;
  int64_t ray_offset;   // the view's rays in the concatenated arrays
  int64_t ray_count;
  int32_t scene;
  int32_t pad;
};

struct BatchFwdParams {
  const BatchScene* scenes;
  const BatchView* views;
  int num_views;
  const int32_t* slot_ray;  // global ray index per slot, -1 for padding
  int64_t num_slots;
  const float* rayo;
  const float* rayd;
  int64_t R;
  float tmin, tmax;
  int max_iters;
  EverForwardOut out;  // ray-indexed outputs; event_log columns are slots (stride num_slots)
  unsigned int* work_counter;
  int grid;            // persistent blocks
  int frustum;         // frustum phase before the rounds (set from the tune)
  int stack_depth;     // traversal stack entries in use (set from the tune)
};

cudaError_t launch_forward_batched(const BatchFwdParams& P, int deg, const EverTune& tune, cudaStream_t st);
template <int KBUF>
cudaError_t launch_forward_batched_k(const BatchFwdParams& P, int deg, int block, cudaStream_t st);

struct BatchBwdParams {
  const BatchScene* scenes;
  const BatchView* views;
  int num_views;
  const int32_t* slot_ray;
  const int32_t* slot_order;  // nullable: packet lane position -> slot (slots of any view)
  int64_t num_slots;
  const float* rayo;
  const float* rayd;
  int64_t R;
  float tmin, tmax;
  int max_iters;
  const float* grad_out;
  const float* states;
  const int32_t* iters;
  const int32_t* event_log;
  int log_cap;
  float* drayo;
  float* drayd;
  unsigned int* work_counter;
  int grid;
};

cudaError_t launch_backward_batched(const BatchBwdParams& P, int deg, const EverTune& tune, cudaStream_t st);

struct BwdParams {
  const void* nodes;
  const void* records;
  const float* features;
  const int32_t* order;
  int64_t N;
  int K;
  const float* rayo;
  const float* rayd;
  int64_t R;
  float tmin, tmax;
  int max_iters;
  const int32_t* ray_order;
  const int32_t* slot_order;  // nullable: launch position -> forward slot
  const float* grad_out;
  const float* states;
  const int32_t* iters;
  const int32_t* event_log;
  int log_cap;
  const float* wct;
  int num_wct;
  float* acc_geo;   // N x 16 (W 9, mean 3, density 1, DC feature gradient 3 at degree 0), Morton order
  float* acc_feat;  // N x K x 3, Morton order
  float* dmeans2d;  // per-ray wct mode accumulates here directly (original order)
  float* drayo;
  float* drayd;
};

cudaError_t launch_backward(const BwdParams& P, int deg, const EverTune& tune, cudaStream_t st);

struct FinalizeParams {
  const void* records;
  const int32_t* order;
  int64_t N;
  int K;
  const float* mean;
  const float* scale;
  const float* quat;
  const float* acc_geo;
  const float* acc_feat;
  int32_t* inv_order;  // (N) scratch: Morton position of each original index
  bool dc_only;      // degree-0 trace: acc_feat was neither cleared nor written (not read)
  const float* wct;  // first matrix, for the single-camera dmeans2d
  int num_wct;
  EverBackwardOut out;
};

cudaError_t launch_finalize(const FinalizeParams& P, cudaStream_t st);
cudaError_t launch_log_to_reference(const int32_t* order, const int32_t* log, int log_cap, const int32_t* iters,
                                    int64_t R, const int32_t* ray_order, int32_t* tri, int max_iters, cudaStream_t st);

// ---- ray-cost model (39 -> 64 -> 64 -> 2 MLP on the tensor cores) ----
// fp32 parameter block: W1 [64 x 64], W2 [64 x 64], W3 [16 x 64] (row = output unit), then
// b1 [64], b2 [64], b3 [16]. Input columns 39..63 of W1 and output rows 2..15 of W3 pad the
// shapes to the MMA tile and stay zero.
constexpr int kOffW1 = 0, kOffW2 = 4096, kOffW3 = 8192, kOffB1 = 9216, kOffB2 = 9280, kOffB3 = 9344;
constexpr int kMlpParams = 9360;
constexpr int kMlpMaxGrid = 160;  // CTAs of a gradient launch (one partial-gradient slot each)

struct MlpParams {
  const void* w1;  // bf16 [64 x 64]
  const void* w2;  // bf16 [64 x 64]
  const void* w3;  // bf16 [16 x 64]
  const float* params;
  const float* rayo;  // rays to encode, or
  const float* rayd;
  const float* feat;  // pre-encoded inputs (num x 64 fp32), used instead of the rays when set
  const int32_t* sample_idx;  // sample s reads ray sample_idx[s] (nullable: s)
  int64_t num_samples;
  float cx, cy, cz, inv_scale;  // scene centre and 1 / scale of the encoding
  // inference
  float* pred;     // (rays, 2), indexed by ray
  uint8_t* bins;   // nullable: cost bin of each ray from pred[.,0] and the thresholds
  float thr[3];
  // training
  const float* target;  // (rays, 2)
  float loss_w0, loss_w1, inv_batch;
  float* partial;  // (grid, kMlpParams + 1): per-CTA gradient and loss
  int32_t* error;  // set to 1 when a tensor-core wait times out
  long long wait_clocks;  // bound of each tensor-core completion wait (0: about a second)
};

// One persistent CTA per SM at most; `grid` from mlp_grid.
cudaError_t launch_mlp(const MlpParams& P, bool train, int grid, cudaStream_t st);
int mlp_grid(int64_t num_samples, int max_grid, bool train);
cudaError_t launch_mlp_reduce(const float* partial, int grid, float* grads, float* loss, cudaStream_t st);
cudaError_t launch_mlp_adam(float* params, const float* grads, float* m, float* v, void* w1, void* w2, void* w3,
                            float lr, float beta1, float beta2, float eps, int step, cudaStream_t st);
cudaError_t launch_mlp_pack(const float* params, void* w1, void* w2, void* w3, cudaStream_t st);

// ---- colour pre-pass and camera rays (shprep.cu) ----
// grad_out == nullptr: forward (out = colour or features); else backward (out = grad_features).
cudaError_t launch_sh_prepass(const float* mean, const float* feat, int64_t N, int K, int deg, const float* cam,
                              int mode, const float* grad_out, float* out, cudaStream_t st);

struct CameraParams {
  int width, height;
  float fx, fy, cx, cy;
  float c2w[12];
};
cudaError_t launch_camera_rays(const CameraParams& C, const float* jitter, float* rayo, float* rayd, cudaStream_t st);

// Camera traces (rays made in the kernels; slots of 8x4 pixel tiles, camera.cuh).
cudaError_t launch_forward_camera(const FwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                  const EverTune& tune, cudaStream_t st);
template <int KBUF>
cudaError_t launch_forward_camera_k(const FwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                    int block, cudaStream_t st);
// Backward of a camera trace: P.R is the slot count, P.slot_order (nullable) the launch
// order over slots, P.ray_order unused; drayo/drayd (nullable) are indexed by pixel.
cudaError_t launch_backward_camera(const BwdParams& P, const CameraParams& cam, const float* jitter, int deg,
                                   const EverTune& tune, cudaStream_t st);
cudaError_t camera_backward_slot_order(const CameraParams& cam, const int32_t* iters, int shift, char* ws,
                                       int32_t* slot_order, cudaStream_t st);
cudaError_t launch_camera_slot_pixels(const CameraParams& cam, int32_t* slot_pixel, cudaStream_t st);
cudaError_t launch_camera_log_to_reference(const CameraParams& cam, const int32_t* order, const int32_t* log,
                                           int log_cap, const int32_t* iters, int32_t* tri, int max_iters,
                                           cudaStream_t st);

}  // namespace ever
