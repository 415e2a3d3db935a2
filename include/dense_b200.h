/* dense_b200.h: C ABI of the B200 dense depthmap library (libdense_b200.so).
 *
 * Drop-in for the legacy pydense classes of OpenSfM's dense path
 * (opensfm/src/lib/dense/depthmap.h:57-153, Python surface in
 * opensfm/src/lib/dense/pydense.pyi:28-77).  Plain pointers and sizes only.
 *
 * Conventions
 *  - Matrices are row-major float64: K, R are 3x3 (9 doubles), t is 3.
 *    Cameras map world X to x_cam = R X + t, pixels q ~ K x_cam.
 *  - Images and masks are uint8 H x W, row-major, `stride` bytes per row
 *    (stride >= width).  View 0 of an estimator/cleaner/pruner is the
 *    reference view, as in the reference classes.
 *  - Outputs are caller-owned host buffers: depth f32 [H][W], plane f32
 *    [H][W][3] (plane v with v.X + 1 = 0 in reference-camera coordinates),
 *    score f32 [H][W], nghbr i32 [H][W].
 *  - Inputs are copied (to device memory) by add_view; callers may free
 *    them afterwards (depthmap.cc:156-157, 521, 571-574 copy too).
 *  - Every call returns a dn_status; on failure dn_last_error() gives a
 *    message (thread-local).  Nothing here aborts or traps.
 *  - Each object owns one CUDA stream; calls on one object are serialised
 *    by the caller, different objects may be used from different threads.
 */
#ifndef DENSE_B200_H_
#define DENSE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DN_OK = 0,
  DN_INVALID_ARG = 1,    /* bad size, shape, count or parameter value */
  DN_OUT_OF_MEMORY = 2,  /* device or pinned allocation failed */
  DN_DEVICE_ERROR = 3,   /* CUDA runtime error, or no usable device */
  DN_TIMEOUT = 4,        /* a bounded device-side wait expired */
  DN_NOT_READY = 5,      /* result requested before it was computed */
  DN_OUT_OF_RANGE = 6    /* an index out of range (the reference throws std::out_of_range) */
} dn_status;

/* Message for the last failed call on this thread ("" if none). */
const char* dn_last_error(void);
/* Library version string. */
const char* dn_version(void);
/* Number of visible CUDA devices (0 if none). */
int dn_device_count(void);
/* Makes `device` current for this thread; objects created afterwards on
 * this thread live on it. */
dn_status dn_set_device(int device);

/* ------------------------------------------------------------------------
 * DepthmapEstimator (depthmap.h:57-111; pydense.pyi:45-60)
 * ---------------------------------------------------------------------- */
typedef struct dn_estimator dn_estimator;

/* DepthmapEstimator::DepthmapEstimator (depthmap.cc:134-144): patch 7,
 * 50 planes, 3 iterations, min patch sd 5. */
dn_status dn_estimator_create(dn_estimator** out);
dn_status dn_estimator_destroy(dn_estimator* est);
/* DepthmapEstimator::AddView (depthmap.cc:146-162).  mask may be NULL (all
 * valid).  The first view is the reference and sets the output size; the
 * other views may have any size (each is sampled with its own extent, as in
 * depthmap.cc:472). */
dn_status dn_estimator_add_view(dn_estimator* est, const double* K, const double* R,
                                const double* t, const uint8_t* image, const uint8_t* mask,
                                int width, int height, int stride);
/* SetDepthRange (depthmap.cc:164-169). */
dn_status dn_estimator_set_depth_range(dn_estimator* est, double min_depth, double max_depth,
                                       int num_depth_planes);
/* SetPatchMatchIterations (depthmap.cc:171-173). */
dn_status dn_estimator_set_patchmatch_iterations(dn_estimator* est, int n);
/* SetPatchSize (depthmap.cc:175-178).  Supported: 3 <= size <= 12
 * (half-size 1..5). */
dn_status dn_estimator_set_patch_size(dn_estimator* est, int size);
/* SetMinPatchSD (depthmap.cc:180-182): stores sd * sd. */
dn_status dn_estimator_set_min_patch_sd(dn_estimator* est, float sd);
/* Seed of the counter-based RNG used by PatchMatch (no counterpart: the
 * reference seeds std::mt19937 from std::random_device). */
dn_status dn_estimator_set_seed(dn_estimator* est, uint64_t seed);

/* ComputeBruteForce (depthmap.cc:184-200). */
dn_status dn_estimator_compute_brute_force(dn_estimator* est, float* depth, float* plane,
                                           float* score, int32_t* nghbr);
/* ComputePatchMatch (depthmap.cc:202-213), red-black schedule. */
dn_status dn_estimator_compute_patch_match(dn_estimator* est, float* depth, float* plane,
                                           float* score, int32_t* nghbr);
/* ComputePatchMatchSample (depthmap.cc:215-227), red-black schedule. */
dn_status dn_estimator_compute_patch_match_sample(dn_estimator* est, float* depth,
                                                  float* plane, float* score, int32_t* nghbr);
/* ComputePlaneScore (depthmap.cc:408-419) for every interior pixel with the
 * caller's planes (f32 [H][W][3]); border pixels get score 0, nghbr 0. */
dn_status dn_estimator_score_planes(dn_estimator* est, const float* planes, float* score,
                                    int32_t* nghbr);
/* PatchMatch from a caller-supplied initial plane field (f32 [H][W][3];
 * planes with z == 0 fall back to the random initialisation of
 * RandomInitialization, depthmap.cc:237-256).  Used by the learned proposal. */
dn_status dn_estimator_compute_patch_match_init(dn_estimator* est, const float* init_planes,
                                                float* depth, float* plane, float* score,
                                                int32_t* nghbr);
/* Number of NCC taps the last compute evaluated (device counter). */
dn_status dn_estimator_last_taps(dn_estimator* est, uint64_t* taps);

/* ------------------------------------------------------------------------
 * DepthmapCleaner (depthmap.h:113-129; pydense.pyi:28-42)
 * ---------------------------------------------------------------------- */
typedef struct dn_cleaner dn_cleaner;

/* DepthmapCleaner::DepthmapCleaner (depthmap.cc:504-505): threshold 0.01,
 * min consistent views 2. */
dn_status dn_cleaner_create(dn_cleaner** out);
dn_status dn_cleaner_destroy(dn_cleaner* c);
dn_status dn_cleaner_set_same_depth_threshold(dn_cleaner* c, float t);  /* depthmap.cc:507-509 */
dn_status dn_cleaner_set_min_consistent_views(dn_cleaner* c, int n);    /* depthmap.cc:511-513 */
/* DepthmapCleaner::AddView (depthmap.cc:515-522).  depth: f32, row stride
 * in floats (>= width). */
dn_status dn_cleaner_add_view(dn_cleaner* c, const double* K, const double* R, const double* t,
                              const float* depth, int width, int height, int stride);
/* DepthmapCleaner::Clean (depthmap.cc:524-555): out f32 [H][W]. */
dn_status dn_cleaner_clean(dn_cleaner* c, float* clean_depth);

/* ------------------------------------------------------------------------
 * DepthmapPruner (depthmap.h:131-153; pydense.pyi:63-77)
 * ---------------------------------------------------------------------- */
typedef struct dn_pruner dn_pruner;

/* DepthmapPruner::DepthmapPruner (depthmap.cc:557): threshold 0.01. */
dn_status dn_pruner_create(dn_pruner** out);
dn_status dn_pruner_destroy(dn_pruner* p);
dn_status dn_pruner_set_same_depth_threshold(dn_pruner* p, float t);  /* depthmap.cc:559-561 */
/* DepthmapPruner::AddView (depthmap.cc:563-575): depth f32 [H][W], plane
 * f32 [H][W][3], color u8 [H][W][3], label u8 [H][W] (tightly packed). */
dn_status dn_pruner_add_view(dn_pruner* p, const double* K, const double* R, const double* t,
                             const float* depth, const float* plane, const uint8_t* color,
                             const uint8_t* label, int width, int height);
/* DepthmapPruner::Prune (depthmap.cc:577-637), first call: runs the pruner
 * and returns the number of kept points in *count. */
dn_status dn_pruner_prune(dn_pruner* p, int64_t* count);
/* Second call: copies the kept points (row-major pixel order, as the
 * reference appends them) into caller buffers sized for `capacity` points:
 * points f32 [n][3], normals f32 [n][3], colors u8 [n][3], labels u8 [n]. */
dn_status dn_pruner_fetch(dn_pruner* p, float* points, float* normals, uint8_t* colors,
                          uint8_t* labels, int64_t capacity);

/* ------------------------------------------------------------------------
 * Batched reconstruction (no reference counterpart: opensfm/dense.py runs
 * one estimator per reference view; this runs every depthmap of a
 * reconstruction, with mixed image sizes and neighbour counts, in one
 * persistent launch per stage, replayed from a captured CUDA graph).
 * ---------------------------------------------------------------------- */
typedef struct dn_batch dn_batch;

dn_status dn_batch_create(dn_batch** out);
dn_status dn_batch_destroy(dn_batch* b);
/* Uploads one view (image copied to device as FP16).  Views may differ in
 * size.  *view_id receives the view's index. */
dn_status dn_batch_add_view(dn_batch* b, const double* K, const double* R, const double* t,
                            const uint8_t* image, const uint8_t* mask, int width, int height,
                            int stride, int* view_id);
/* Declares one depthmap: reference view, its matching views (used for
 * scoring, <= 16) and its depth range.  *map_id receives its index. */
dn_status dn_batch_add_depthmap(dn_batch* b, int ref_view, const int* matching_views,
                                int n_matching, double min_depth, double max_depth,
                                int* map_id);
/* Cleaner / pruner views of a depthmap (<= 16 other maps by map id); when
 * set, dn_batch_run also cleans (and prunes) after PatchMatch. */
dn_status dn_batch_set_clean_views(dn_batch* b, int map_id, const int* other_maps, int n);
dn_status dn_batch_set_params(dn_batch* b, int patch_size, float min_patch_sd, int iterations,
                              float same_depth_threshold, int min_consistent_views,
                              uint64_t seed);
/* Flags for dn_batch_run. */
#define DN_RUN_CLEAN 1u  /* run the cleaner after PatchMatch */
#define DN_RUN_PRUNE 2u  /* run the pruner after the cleaner */
#define DN_RUN_GRAPH 4u  /* capture the run in a CUDA graph once, replay after */
#define DN_RUN_INIT 8u   /* initialise from planes set by dn_batch_set_init */
#define DN_RUN_TIMING 16u /* record CUDA events around each stage */
/* Learned initialisation: the feature sweep, the proposal network set by
 * dn_batch_set_proposal_net and the plane install run on the batch stream
 * before PatchMatch (inside the graph with DN_RUN_GRAPH); every pixel with
 * a proposal starts from it, the others from the random initialisation. */
#define DN_RUN_LEARNED 32u
/* Enqueues PatchMatch for every declared depthmap (and clean/prune per
 * flags) on the batch's stream; returns without waiting. */
dn_status dn_batch_run(dn_batch* b, unsigned flags);
dn_status dn_batch_synchronize(dn_batch* b);
/* Copies one depthmap's results to host buffers (after synchronize); any
 * pointer may be NULL to skip it.  clean may be NULL. */
dn_status dn_batch_get_depthmap(dn_batch* b, int map_id, float* depth, float* plane,
                                float* score, int32_t* nghbr, float* clean);
/* The final (clean = 0) or cleaned (clean = 1) depth of n maps into host
 * buffers depths[k] (f32 [H][W] of map map_ids[k]), with one stream
 * synchronisation for all of them (no reference counterpart; the copies
 * run asynchronously when the buffers are pinned). */
dn_status dn_batch_get_depths(dn_batch* b, int n, const int* map_ids, float* const* depths,
                              int clean);
/* PatchMatch schedule: half-passes per run (-1: 2 x iterations), and per
 * half-pass the candidate sets: the 4 adjacent planes (use_near), the 4 far
 * planes (use_far), n_refine refinements whose first depth / normal-slope
 * ranges are depth_range0 / normal_range0, shrinking by 0.3 / 0.8 per step.
 * Defaults 1, 1, 6, 0.02, 0.5 follow PatchMatchUpdatePixel
 * (depthmap.cc:305-374). */
dn_status dn_batch_set_schedule(dn_batch* b, int half_passes, int use_near, int use_far,
                                int n_refine, float depth_range0, float normal_range0);
/* Views scored per PatchMatch candidate (no reference counterpart as a
 * switch): mode 0 scores every matching view and keeps the maximum
 * (ComputePlaneScore, depthmap.cc:408-419), as ComputePatchMatch does; mode
 * 1 initialises with every view, then the half-passes score one view per
 * candidate -- the view the candidate's source pixel found best, the
 * current view for refinements -- plus one random other view of the
 * current plane per update; mode 2 is ComputePatchMatchSample
 * (depthmap.cc:215-227, 305-374): a random view at the initialisation, then
 * as mode 1. */
dn_status dn_batch_set_candidate_views(dn_batch* b, int mode);
/* Knight-move candidates (no reference counterpart): with on = 1 each
 * half-pass update also tries the planes of the 8 pixels at (+-1, +-2) and
 * (+-2, +-1), which have the opposite red-black colour. */
dn_status dn_batch_set_knight_moves(dn_batch* b, int on);
/* Active pixels (no reference counterpart): with on = 1, from the third
 * half-pass of a run on, a pixel is updated only if its own depth or one of
 * its 4 neighbours' depths moved at their last update -- by more than
 * min_change relative, or, with min_change = 0, any change of the plane;
 * the others keep their state. */
dn_status dn_batch_set_active_pixels(dn_batch* b, int on, float min_change);
/* How the active half-passes run (separate launches per stage; the
 * persistent launch always takes the second way): on = 1 (default) lists
 * the active pixels of each map and runs the half-pass over the lists; on =
 * 0 runs every tile that holds an active pixel.  The maps are the same. */
dn_status dn_batch_set_active_lists(dn_batch* b, int on);
/* Settled start for active pixels: with min_score > 0 the initialisation
 * marks as moved only the pixels whose initial score is below min_score,
 * and the active rule applies from the first half-pass, so a pixel whose
 * initial plane scores well is updated only once a neighbour moves.
 * min_score = 0 (the default): every pixel starts as moved and the first
 * two half-passes update every pixel. */
dn_status dn_batch_set_active_seed(dn_batch* b, float min_score);
/* The random initialisation as the fallback of given planes (learned
 * proposals or dn_batch_set_init): with on = 1 every pixel with a given
 * plane also draws the reference's random plane (RandomInitialization,
 * depthmap.cc:237-256) and keeps whichever scores higher on the same
 * view(s), the given one on a tie.  Default 0: the given plane. */
dn_status dn_batch_set_init_fallback(dn_batch* b, int on);
/* Initial planes (f32 [H][W][3], reference camera) for one depthmap. */
dn_status dn_batch_set_init(dn_batch* b, int map_id, const float* planes);
/* Total kept pruner points over all maps of the last run (after sync). */
dn_status dn_batch_pruned_count(dn_batch* b, int64_t* count);
/* One map's pruner output of the last DN_RUN_PRUNE run (after sync): the
 * cleaned depth and PatchMatch planes of the map and of its cleaner maps go
 * through DepthmapPruner::Prune (depthmap.cc:577-637), colour = the view's
 * gray level, label 0.  *count receives the point count; buffers (any may
 * be NULL) hold `capacity` points. */
dn_status dn_batch_get_points(dn_batch* b, int map_id, float* points, float* normals,
                              uint8_t* colors, uint8_t* labels, int64_t capacity, int64_t* count);
/* NCC taps evaluated by the last run (device counter). */
dn_status dn_batch_last_taps(dn_batch* b, uint64_t* taps);
/* Replaces the pixels of an uploaded view (same size), asynchronously on
 * the batch stream; the host buffer must stay valid until the next
 * dn_batch_synchronize. */
dn_status dn_batch_set_view_image(dn_batch* b, int view_id, const uint8_t* image, int stride);
/* Pipelined batch I/O (no reference counterpart).  Both calls return at
 * once, and every run gives the same results as with
 * dn_batch_set_view_image / dn_batch_get_depths at the same points of the
 * call sequence.  Their host copies run on two more streams of the batch
 * (uploads, readbacks), so they overlap a run enqueued before (uploads) or
 * after (readbacks); the views uploaded since the last run are prepared
 * (FP16 image, coefficient table) together, in one launch, by the next
 * call that reads views (dn_batch_run, dn_batch_sweep_features,
 * dn_batch_set_view_image).  Host buffers must be pinned for the overlap
 * (pageable ones work, with the copy done before the call returns) and stay
 * valid, and unmodified for an upload, until dn_batch_synchronize; the timer
 * events (dn_batch_timer_record) include these copies.
 *
 * upload_view_image: the pixels of view view_id for runs enqueued after
 * the call.
 * get_depths_async: the final (clean = 0) or cleaned (clean = 1) depth of n
 * maps, as left by the runs enqueued before the call, into depths[k] (f32
 * [H][W] of map map_ids[k]); complete after dn_batch_synchronize. */
dn_status dn_batch_upload_view_image(dn_batch* b, int view_id, const uint8_t* image, int stride);
dn_status dn_batch_get_depths_async(dn_batch* b, int n, const int* map_ids, float* const* depths,
                                    int clean);
/* Per-stage device times (ms) of the last run made with DN_RUN_TIMING:
 * out[0] init, out[1] all PatchMatch half-passes, out[2] post-process,
 * out[3] cleaner and pruner, out[4] whole run, out[5] the learned proposal
 * (sweep, network and plane install; 0 without DN_RUN_LEARNED, and not part
 * of out[0]).  taps_out (may be NULL) receives the NCC taps of init
 * (taps_out[0]) and of the half-passes (taps_out[1]). */
dn_status dn_batch_last_timings(dn_batch* b, float* out, int n, uint64_t* taps_out);
/* Launch tuning (no reference counterpart): thread block shape bx x by
 * (bx * by <= 128, bx a multiple of 32); variant = the lanes that share one
 * pixel in the initialisation and PatchMatch kernels (1, 2, 4 or 8; 2, 4
 * and 8 apply to the 7 x 7 patch), plus 16 to run initialisation, every
 * half-pass and the post-process of all depthmaps in ONE cooperative persistent
 * launch (32 x 4 blocks, 7 x 7 patch; tiles taken from atomic counters,
 * bounded grid barriers between stages).  Chosen by opensfm_b200.autotune;
 * scores agree between settings to float rounding of the sums. */
dn_status dn_batch_set_tuning(dn_batch* b, int bx, int by, int variant);
dn_status dn_estimator_set_tuning(dn_estimator* est, int bx, int by, int variant);
/* Device timer on the batch stream: record event `slot` (0 or 1), and the
 * elapsed ms between the two recorded events (after dn_batch_synchronize). */
dn_status dn_batch_timer_record(dn_batch* b, int slot);
dn_status dn_batch_timer_elapsed(dn_batch* b, float* ms);
/* Copies one depthmap's final depth to a device buffer (no host copy). */
dn_status dn_batch_copy_depth_device(dn_batch* b, int map_id, float* d_out);

/* ------------------------------------------------------------------------
 * Utilities (no reference counterpart)
 * ---------------------------------------------------------------------- */
/* PostProcess (depthmap.cc:489-502) on a host depth map: 5x5 median with
 * replicated borders, then zero where |d - median| / d > 0.05 or d == 0. */
dn_status dn_postprocess_depth(const float* depth, float* out, int width, int height);
/* Check of the bounded device-side waits (no reference counterpart): runs
 * the persistent launch's grid barrier on `blocks` blocks (1..64) with a
 * barrier that can never open (it expects one block more), each block
 * polling at most max_spins times (about 100 ns apart; 1..2^24).  Returns
 * DN_TIMEOUT -- the status every persistent run reports when one of its
 * waits expires -- with the device time in *ms (may be NULL); the device
 * stays usable. */
dn_status dn_check_bounded_wait(int blocks, int64_t max_spins, float* ms);
/* Measures the device's FP32 FMA throughput (TFLOP/s, FMA = 2 flops) with a
 * register-resident FMA loop on every SM; used as the scoring roofline. */
dn_status dn_fp32_peak(double* tflops, double* ms);
/* Measures the ceiling of the scoring walk (no reference counterpart): G
 * taps/s of 7 x 7 affine walks through the FP16 coefficient table with the
 * production sampler and the three weighted NCC sums, one thread per pixel
 * of a 1024 x 768 view, and nothing else (no candidate generation, warp
 * setup, lane groups or NCC finish); the half-pass's tap rate over it is the
 * share of the walk's own ceiling it reaches. */
dn_status dn_walk_ceiling(double* gtaps, double* ms);

/* ------------------------------------------------------------------------
 * Learned initialisation (no reference counterpart: the reference draws the
 * PatchMatch initialisation at random, depthmap.cc:237-256).  A 6-layer 3x3
 * convolutional network (32 channels, BF16 activations, FP32 accumulation,
 * tensor cores) maps per-pixel features (reference intensity + NCC of up
 * to 15 swept fronto-parallel planes against the 2 nearest matching views) to
 * (inverse-depth fraction, normal slopes).  Activations are NHWC BF16 device
 * buffers; `stream` is a cudaStream_t (NULL: default stream); every call
 * enqueues work and returns.
 * ---------------------------------------------------------------------- */
/* Network input features (n_planes planes, 1..15) of every depthmap of the
 * batch on the grid of every `stride`-th pixel (1, 2, 4 or 8; grid point (ys, xs) is pixel
 * (stride ys, stride xs), grid size ceil(W / stride) x ceil(H / stride)):
 * feat is a device BF16 buffer [n_maps][Hs][Ws][32] with map stride
 * `map_stride` elements (>= Hs * Ws * 32 of the largest map).  Runs on the
 * batch stream. */
dn_status dn_batch_sweep_features(dn_batch* b, void* feat, int64_t map_stride, int n_planes,
                                  int stride);
/* Training targets from the last PatchMatch run on the same grid: target is
 * a device f32 buffer [n_maps][Hs][Ws][4] = (inverse-depth fraction, sx,
 * sy, weight), with weight 1 where the depth is valid and its score >=
 * min_score. */
dn_status dn_batch_targets(dn_batch* b, float* target, int64_t map_stride, float min_score,
                           int stride);
/* The proposal network of DN_RUN_LEARNED runs, copied to the device:
 * weights = BF16 bit patterns of the 6 layers' [cout][9 x 32] matrices one
 * after the other (cout 32 for layers 0-4, 4 for layer 5: 46,080 values),
 * biases = FP32 [32] x 5 then [4] (164 values).  Features are swept with
 * n_planes planes (1..15) on the grid of every `stride`-th pixel (1, 2, 4 or 8),
 * the network runs on that grid (maps of one grid size in one batch) and
 * its output is interpolated back to every pixel.  weights = NULL removes
 * the network. */
dn_status dn_batch_set_proposal_net(dn_batch* b, const uint16_t* weights, const float* biases,
                                    int n_planes, int stride);
/* The larger side (pixels) of the images the network was trained on.  With
 * ref_dim > 0 each map's proposal grid uses the network's stride scaled by
 * the map's larger side over ref_dim, rounded down to 1, 2, 4 or 8, so that
 * every map's grid has the training scale (a 320 x 240 map at stride 2
 * when the network was trained at stride 4 on 640 x 480); ref_dim = 0 (the
 * default): every map uses the stride. */
dn_status dn_batch_set_proposal_scale(dn_batch* b, int ref_dim);
/* Initial planes of one depthmap from the network output (device f32
 * [H][W][4]); the next dn_batch_run with DN_RUN_INIT starts from them. */
dn_status dn_batch_init_from_output(dn_batch* b, int map_id, const float* out);
/* y = act(conv3x3(x, w) + bias) over n_pix pixels of images H x W; relu 0/1;
 * y (BF16) and/or y32 (FP32) may be NULL.  cin 32; cout 32 or 4.  Runs on
 * the tcgen05 tensor cores (implicit GEMM, M = 128 pixels per tile, FP32
 * accumulators in tensor memory); asynchronous on `stream`, errors of its
 * bounded waits are reported by dn_nn_synchronize. */
dn_status dn_nn_conv3x3_forward(const void* x, const void* w, const float* bias, int64_t n_pix,
                                int H, int W, int cin, int cout, int relu, void* y, float* y32,
                                void* stream);
/* The same forward with warp-level mma.sync (m16n8k16) tensor-core
 * instructions, kept for comparison. */
dn_status dn_nn_conv3x3_forward_mma_sync(const void* x, const void* w, const float* bias,
                                         int64_t n_pix, int H, int W, int cin, int cout, int relu,
                                         void* y, float* y32, void* stream);
/* Waits for `stream`; DN_TIMEOUT if a tensor-core wait expired since the
 * last call (the outputs of that launch are then invalid). */
dn_status dn_nn_synchronize(void* stream);
/* Backward of one layer given dy, the gradient of its pre-activation output
 * (BF16 [n_pix][cout]): accumulates dw [cout][9 cin] and db [cout] (FP32,
 * atomic adds) and writes dx (BF16 [n_pix][cin]) multiplied by (x_mask > 0)
 * when x_mask is given, which makes dx the pre-activation gradient of a
 * ReLU layer below whose output x_mask is.  dx may be NULL; wt_scratch holds
 * cin * 9 * 16 * ceil(cout / 16) BF16 values. */
dn_status dn_nn_conv3x3_backward(const void* dy, const void* x, const void* w,
                                 const void* x_mask, int64_t n_pix, int H, int W, int cin,
                                 int cout, void* dx, float* dw, float* db, void* wt_scratch,
                                 void* stream);
/* The same backward on the tcgen05 tensor cores (the training path; the
 * warp-level mma.sync version above is kept as the comparison): dw and db
 * from a split-K GEMM with FP32 accumulators in tensor memory, dx from the
 * forward tcgen05 kernel on dy with flipped weights and the x_mask ReLU
 * mask.  scratch: a device buffer of at least
 * dn_nn_backward_scratch_bytes(n_pix, cout) bytes (16-byte aligned).
 * Bounded waits report through dn_nn_synchronize. */
int64_t dn_nn_backward_scratch_bytes(int64_t n_pix, int cout);
dn_status dn_nn_conv3x3_backward_tc(const void* dy, const void* x, const void* w,
                                    const void* x_mask, int64_t n_pix, int H, int W, int cin,
                                    int cout, void* dx, float* dw, float* db, void* scratch,
                                    int64_t scratch_bytes, void* stream);
/* L1 loss of pred (f32 [n_pix][4]) against target ([n_pix][4], last = weight)
 * with the normal slopes weighted by normal_weight: adds the loss and the
 * weight total to loss_sum[0] / count[0] and writes dpred (BF16 [n_pix][4]). */
dn_status dn_nn_l1_loss(const float* pred, const float* target, int64_t n_pix,
                        float normal_weight, void* dpred, float* loss_sum, float* count,
                        void* stream);
/* Adam step on n FP32 parameters with grad / max(count, 1); also writes the
 * BF16 copy w16 (may be NULL).  bc1 / bc2 are the bias corrections. */
dn_status dn_nn_adam(float* w, float* m, float* v, const float* grad, int n, const float* count,
                     float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                     void* w16, void* stream);

/* ------------------------------------------------------------------------
 * Pruning without device allocation.
 *
 * No counterpart in the reference.  DepthmapPruner::Prune for callers that
 * cannot allocate device memory (their process hands the GPU's memory to its
 * own pool, or must not allocate once running).  Inputs and outputs are
 * caller-owned DEVICE buffers; the working memory is a static array compiled
 * into the library (about 4.3 MB per GPU, held until exit).  Limits: the
 * reference depthmap (view 0) has at most 4,194,304 pixels, at most 17 views,
 * and `capacity` (points the output buffers hold) is at least its
 * width * height; every view is at most 16384 pixels a side, with finite
 * K, R, t and an invertible K (as dn_pruner_add_view checks).  The number of
 * kept points is written to the device counter *count.  Work is enqueued on
 * `stream` (a cudaStream_t, NULL for the default stream), the view table
 * included (it is passed as a kernel argument, so the host array `views`
 * may be freed on return), and the call returns without waiting.  All calls share
 * the static array: calls whose GPU work overlaps race and must be
 * serialised by the caller.  The first call on a device looks up the array's
 * address with that device current; make it before any stream capture.
 * ---------------------------------------------------------------------- */
typedef struct {
  double K[9], R[9], t[3];  /* host values, as for dn_pruner_add_view */
  const float* depth;       /* device, [height][width] */
  const float* plane;       /* device, [height][width][3] */
  const uint8_t* color;     /* device, [height][width][3] */
  const uint8_t* label;     /* device, [height][width] */
  int width, height;
} dn_prune_view;

dn_status dn_prune_noalloc(const dn_prune_view* views, int n_views, float same_depth_threshold,
                           float* points, float* normals, uint8_t* colors, uint8_t* labels,
                           int64_t capacity, unsigned long long* count, void* stream);
/* Message for the last failed dn_prune_noalloc call on this thread. */
const char* dn_noalloc_last_error(void);

/* ----------------------------------------------------------------------
 * GPUDepthmapCleaner (cleaner.h:16-60, cleaner.cc:19-170; kernel
 * acmmp_clean_depthmap, opencl_kernels.h:2155-2273): per reference pixel,
 * forward reprojection into each source (at most 16), space carving (a
 * source seeing farther than (1 + carving_threshold) x the point carves it),
 * and a backward check (the source's point projects back within 2 px and
 * the threshold).  Keep if consistent views (counting the reference) >=
 * min(min_consistent_views, 1 + neighbours) and carved < max_carved_views.
 * FP32 in the kernel's operation order; the source depth is sampled
 * bilinearly with exact fractions.  Sources must have the reference's size.
 * Defaults: threshold 0.01, 3 views, carving 0.2, 1 carved view.
 * ---------------------------------------------------------------------- */
typedef struct dn_gpu_cleaner dn_gpu_cleaner;
dn_status dn_gpu_cleaner_create(dn_gpu_cleaner** out);
dn_status dn_gpu_cleaner_destroy(dn_gpu_cleaner* c);
dn_status dn_gpu_cleaner_set_same_depth_threshold(dn_gpu_cleaner* c, float t);
dn_status dn_gpu_cleaner_set_min_consistent_views(dn_gpu_cleaner* c, int n);
dn_status dn_gpu_cleaner_set_carving_threshold(dn_gpu_cleaner* c, float t);
dn_status dn_gpu_cleaner_set_max_carved_views(dn_gpu_cleaner* c, int n);
/* The device the cleaner's views and kernels live on (default: the current
 * device at create).  Keeps the settings above.  Only before the first
 * add_view, or after dn_gpu_cleaner_clear; DN_INVALID_ARG otherwise. */
dn_status dn_gpu_cleaner_set_device(dn_gpu_cleaner* c, int device);
/* AddView (cleaner.cc:39-54): depth f32 [height][stride]; *id (may be NULL)
 * receives the view index. */
dn_status dn_gpu_cleaner_add_view(dn_gpu_cleaner* c, const double K[9], const double R[9],
                                  const double t[3], const float* depth, int width, int height,
                                  int stride, int* id);
/* Clean (cleaner.cc:56-170): the cleaned depth of view `ref` against
 * `neighbor_ids` into out (f32 [H][W] of the reference view).
 * DN_OUT_OF_RANGE for an index out of range. */
dn_status dn_gpu_cleaner_clean(dn_gpu_cleaner* c, int ref, const int* neighbor_ids, int n,
                               float* out);
/* Clear (cleaner.cc:172-184): removes every view. */
dn_status dn_gpu_cleaner_clear(dn_gpu_cleaner* c);

/* ----------------------------------------------------------------------
 * DepthmapFuser (fuser.h:28-77, fuser.cc:35-482): per-pixel fusion of
 * depthmaps into points, the reference's single-thread order (primary views
 * in order, pixels in raster order, fused pixels marking themselves and the
 * source pixels they used).  The candidate observations of every pixel and
 * the medians are computed on the GPU, the marks on the host.  FP32 in the
 * reference's expression order.  Then the statistical outlier removal
 * (fuser.cc:374-482): exact mean distance to the K nearest other points on
 * the GPU (uniform grid), mean + factor x std threshold on the host.
 * Defaults: 3 consistent observations, 2 px, 0.01, 10 degrees, border 5,
 * behind factor 0.3, outlier removal with K = 12 and factor 2.5.
 * ---------------------------------------------------------------------- */
typedef struct dn_fuser dn_fuser;
dn_status dn_fuser_create(dn_fuser** out);
dn_status dn_fuser_destroy(dn_fuser* f);
dn_status dn_fuser_set_min_num_consistent(dn_fuser* f, int n);
dn_status dn_fuser_set_max_reproj_error(dn_fuser* f, float px);
dn_status dn_fuser_set_max_depth_error(dn_fuser* f, float ratio);
dn_status dn_fuser_set_max_normal_error(dn_fuser* f, float degrees);
dn_status dn_fuser_set_border_margin(dn_fuser* f, int px);
/* SetSORParams (fuser.cc:66-69): knn <= 0 skips the outlier removal;
 * knn above 64 is rejected (DN_INVALID_ARG). */
dn_status dn_fuser_set_sor_params(dn_fuser* f, int knn, float stddev_factor);
dn_status dn_fuser_set_behind_depth_factor(dn_fuser* f, float factor);
/* AddView (fuser.cc:82-97): depth f32 [H][W], normal f32 [H][W][3] (camera
 * frame), color u8 [H][W][3], mask u8 [H][W] or NULL (0 = invalid), the
 * indices of the views to check against, and whether the view is fused. */
dn_status dn_fuser_add_view(dn_fuser* f, const double K[9], const double R[9], const double t[3],
                            const float* depth, const float* normal, const uint8_t* color,
                            const uint8_t* mask, int width, int height, const int* neighbor_ids,
                            int n_neighbors, int primary);
/* Fuse (fuser.cc:115-482): *count receives the number of fused points
 * left after the outlier removal. */
dn_status dn_fuser_fuse(dn_fuser* f, int64_t* count);
/* The last fuse's points, unit normals (world frame) and colours, each
 * `capacity` >= count rows of 3; any pointer may be NULL. */
dn_status dn_fuser_get(dn_fuser* f, float* points, float* normals, uint8_t* colors,
                       int64_t capacity);
/* Device time (ms) of the last fuse's outlier removal; 0 when skipped. */
dn_status dn_fuser_last_removal_ms(dn_fuser* f, float* ms);
/* The fuser's statistical outlier removal on any points (xyz rows, n of
 * them): keep[i] = 1 for points whose mean distance to their knn nearest
 * other points is at most mean + factor x std of those means; mean_knn
 * (may be NULL) receives the means.  knn <= 0 or n <= knn + 1 keeps all
 * (as the reference skips the step); knn above 64 is rejected.  Runs on the
 * current device; errors are reported by dn_fuser_last_error. */
dn_status dn_sor_filter(const float* points, int64_t n, int knn, float stddev_factor,
                        uint8_t* keep, float* mean_knn);
/* Message for the last failed dn_fuser_* or dn_sor_filter call on this
 * thread. */
const char* dn_fuser_last_error(void);

/* ----------------------------------------------------------------------
 * SVOFuser (svo_fuser.h:14-68, svo_fuser.cc:12-183; kernels
 * svo_opencl_kernels.h:187-651): TSDF fusion of depthmaps into a sparse
 * voxel hash (one 64-bit key per voxel, fixed-point integer sums), then
 * surface points where the TSDF changes sign between a voxel and its +X,
 * +Y or +Z neighbour.  Points come in ascending voxel order (x, y, z
 * signed), +X, +Y, +Z per voxel.  FP32 in the kernel source's order.
 * Defaults: voxel 0.02, truncation 4 voxels, minimum weight 3.
 * ---------------------------------------------------------------------- */
typedef struct dn_svo dn_svo;
dn_status dn_svo_create(dn_svo** out);
dn_status dn_svo_destroy(dn_svo* f);
/* SetVoxelSize / SetTruncFactor / SetMinWeight (svo_fuser.cc:15-21),
 * clamped to >= 1e-6, >= 1, >= 0 as the reference does. */
dn_status dn_svo_set_voxel_size(dn_svo* f, float size);
dn_status dn_svo_set_trunc_factor(dn_svo* f, float factor);
dn_status dn_svo_set_min_weight(dn_svo* f, float w);
/* SetDevice (svo_fuser.cc:23): before the first add_view. */
dn_status dn_svo_set_device(dn_svo* f, int device);
/* SetBBox (svo_fuser.cc:25-31): clip to the voxels of [min, max] (world). */
dn_status dn_svo_set_bbox(dn_svo* f, const float min_world[3], const float max_world[3]);
/* AddView (svo_fuser.cc:37-50): depth f32 [H][W]; normal f32 [H][W][3]
 * (camera frame), color u8 [H][W][3], mask u8 [H][W] (0 = skip), weight
 * f32 [H][W] (confidence): each may be NULL. */
dn_status dn_svo_add_view(dn_svo* f, const double K[9], const double R[9], const double t[3],
                          const float* depth, const float* normal, const uint8_t* color,
                          const uint8_t* mask, const float* weight, int width, int height);
/* CountVoxels (svo_fuser.cc:52-106): distinct voxels the views' truncation
 * bands touch; 0 without views. */
dn_status dn_svo_count_voxels(dn_svo* f, uint32_t* count);
/* Fuse (svo_fuser.cc:108-183): *count receives the number of points.
 * DN_INVALID_ARG if there are views but count_voxels has not run. */
dn_status dn_svo_fuse(dn_svo* f, int64_t* count);
/* The last fuse's points, unit normals and colours (rows of 3). */
dn_status dn_svo_get(dn_svo* f, float* points, float* normals, uint8_t* colors,
                     int64_t capacity);
/* Device time (ms) of the last fuse: integration and extraction. */
dn_status dn_svo_last_fuse_ms(dn_svo* f, float* ms);
/* Message for the last failed dn_svo_* call on this thread. */
const char* dn_svo_last_error(void);

/* ----------------------------------------------------------------------
 * DepthmapClusterEstimator (cluster.h, cluster_estimator.cc:21-147, bound
 * at python/pybind.cc:53-104) over the live path's PatchMatch estimator
 * (estimator.cc:120-243, 664-1040; kernels opencl_kernels.h:44-1124,
 * 1298-2099), with the SfM planar prior.  Levels run coarsest first: images
 * area-downscaled by 2^k (OpenCV's INTER_AREA), each reference initialised
 * randomly on the first level and from its own coarser result above it,
 * with the linked references' previous-level depths in a geometric term.
 * Per level: red/black PatchMatch passes (bilateral NCC over strides 1-3,
 * census fallback, joint view selection, refinement) and a checkerboard
 * median filter per iteration; readback (a 5x5 median rejection on the
 * last level) and a logistic confidence.  FP32 with every operation
 * rounded by itself and the library's own exp / log.
 * Defaults: 3 iterations, patch 11, sigma 5 / (3/255), top-k 4, census
 * weight 0.3, smoothness 0, one level.
 * ---------------------------------------------------------------------- */
typedef struct dn_acmmp dn_acmmp;
dn_status dn_acmmp_create(dn_acmmp** out);
dn_status dn_acmmp_destroy(dn_acmmp* e);
/* DepthmapParams setters (depthmap_bind.h:21-33). */
dn_status dn_acmmp_set_max_iterations(dn_acmmp* e, int n);
dn_status dn_acmmp_set_patch_size(dn_acmmp* e, int size);
dn_status dn_acmmp_set_max_image_size(dn_acmmp* e, int size);
/* Pyramid levels (the reference's default pipeline uses 4). */
dn_status dn_acmmp_set_hierarchy_levels(dn_acmmp* e, int levels);
dn_status dn_acmmp_set_sigma_spatial(dn_acmmp* e, float v);
dn_status dn_acmmp_set_sigma_color(dn_acmmp* e, float v);
dn_status dn_acmmp_set_top_k(dn_acmmp* e, int k);
dn_status dn_acmmp_set_census_weight(dn_acmmp* e, float w);
dn_status dn_acmmp_set_smooth_weight(dn_acmmp* e, float w);
dn_status dn_acmmp_set_geom_consistency_weight(dn_acmmp* e, float w);
dn_status dn_acmmp_set_device(dn_acmmp* e, int device);
/* BeginRefView (cluster_estimator.cc:41-53): image u8 [h][stride]; *ref_idx
 * (may be NULL) receives the reference's index. */
dn_status dn_acmmp_begin_ref_view(dn_acmmp* e, const double K[9], const double R[9],
                                  const double t[3], const uint8_t* image, int width, int height,
                                  int stride, float depth_min, float depth_max, int* ref_idx);
/* AddSourceView (cluster_estimator.cc:55-62): a source of the last reference
 * (at most 16 are used). */
dn_status dn_acmmp_add_source_view(dn_acmmp* e, const double K[9], const double R[9],
                                   const double t[3], const uint8_t* image, int width, int height,
                                   int stride);
/* SetSfMPoints (estimator.cc:108-118): world points (rows of 3) of the last
 * reference; each level projects them, triangulates (Delaunay), fits a
 * plane per triangle and centres the refinement hypotheses of the covered
 * pixels on it (estimator.cc:664-940). */
dn_status dn_acmmp_set_sfm_points(dn_acmmp* e, const double* points, int64_t n);
/* AddGeomLink (cluster_estimator.cc:73-80): above the first level, source
 * `source_view_idx` of `ref_idx` takes `from_ref_idx`'s previous depths. */
dn_status dn_acmmp_add_geom_link(dn_acmmp* e, int ref_idx, int source_view_idx, int from_ref_idx);
/* Run (cluster_estimator.cc:82-138): every reference view in turn. */
dn_status dn_acmmp_run(dn_acmmp* e);
dn_status dn_acmmp_num_refs(dn_acmmp* e, int* n);
dn_status dn_acmmp_result_size(dn_acmmp* e, int ref_idx, int* width, int* height);
/* A reference's result: depth [H][W], normal [H][W][3], cost, confidence;
 * any pointer may be NULL.  DN_OUT_OF_RANGE for a bad index. */
dn_status dn_acmmp_get_result(dn_acmmp* e, int ref_idx, float* depth, float* normal, float* cost,
                              float* confidence);
/* Device time (ms) of the last run's kernels, over all references. */
dn_status dn_acmmp_last_run_ms(dn_acmmp* e, float* ms);
/* Clear (cluster_estimator.cc:140). */
dn_status dn_acmmp_clear(dn_acmmp* e);
/* Message for the last failed dn_acmmp_* call on this thread. */
const char* dn_acmmp_last_error(void);
/* The planar prior's Delaunay triangulation of n points (xy rows of 2)
 * inside [0, w) x [0, h), with cv::Subdiv2D's virtual outer triangle;
 * host only: *count triangles as ascending index triples, sorted, into
 * tris (capacity triangles; NULL to query the count). */
dn_status dn_delaunay_2d(const double* xy, int n, int w, int h, int* tris, int capacity,
                         int* count);

/* ----------------------------------------------------------------------
 * Depthmap files (host only, no GPU needed).  OpenSfM stores each view's
 * raw and cleaned depthmap as an .npz archive wrapped in one LZ4 frame
 * (opensfm/dataset.py:1080-1098 writes with lz4.frame.compress,
 * 1100-1112 reads with lz4.frame.decompress).  These replace that
 * dependency; opensfm_b200/dense_io.py uses them.
 * ---------------------------------------------------------------------- */
/* xxHash32 of n bytes (the LZ4 frame checksums). */
uint32_t dn_xxh32(const void* data, int64_t n, uint32_t seed);
/* Largest frame dn_lz4f_compress can write for n input bytes. */
int64_t dn_lz4f_compress_bound(int64_t n);
/* One LZ4 frame (independent 4 MB blocks, content size stored, stored
 * blocks where compression does not pay): *out_len receives its size; dst
 * may be NULL to query it, else it must hold `capacity` >= *out_len bytes. */
dn_status dn_lz4f_compress(const void* src, int64_t n, void* dst, int64_t capacity,
                           int64_t* out_len);
/* Decodes one or more concatenated LZ4 frames (linked or independent
 * blocks, optional block / content checksums and content size, skippable
 * frames).  Call with dst NULL to get *out_len, then again with the same
 * src and a buffer of at least that many bytes. */
dn_status dn_lz4f_decompress(const void* src, int64_t n, void* dst, int64_t capacity,
                             int64_t* out_len);
/* Message for the last failed depthmap-file call on this thread. */
const char* dn_io_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* DENSE_B200_H_ */
