/*
 * k3dom_b200.h -- C ABI of the B200-native K3DOM / DS-PHD/MIB map-and-track update.
 *
 * The library replaces the GPU update of the K3DOM ROS package: the classes
 * dom::DOM_c (include/common/dom.h:16-148), dom::DOM for K3DOM
 * (include/k3dom/dom.h:17-30) and dom::DOM for DS-PHD/MIB (include/dsphdmib/dom.h:17-37).
 * Both variants live behind one handle type here, chosen at creation time.
 *
 * Conventions
 *  - Every call returns a k3dom_status; nothing is printed and nothing traps.
 *  - A handle is used by one host thread at a time (the caller serialises).
 *  - `mem` arguments say where a caller buffer lives: K3DOM_MEM_HOST or K3DOM_MEM_DEVICE
 *    (device memory of the handle's GPU).
 *  - Particle positions/velocities are in voxel-index units (voxels, voxels/s), exactly as
 *    in the reference (k3dom_node.cpp:352-357). Points are metres, sensor-centred and
 *    map-axis aligned (src/k3dom/kernel/mass_update.cu:96-99).
 *  - Cell index = x + G*y + G*G*z with x fastest (src/common/kernel/predict.cu:52-55).
 *  - Synchronous calls (k3dom_update_grid, the stage calls, the readbacks) return after the
 *    GPU work is complete, as DOM::updateGrid does with cudaDeviceSynchronize
 *    (src/k3dom/dom.cu:47). The *_async forms only enqueue on the handle's stream.
 */
#ifndef K3DOM_B200_H
#define K3DOM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define K3DOM_B200_ABI_VERSION 2

typedef enum k3dom_status {
    K3DOM_OK = 0,
    K3DOM_ERR_INVALID_ARGUMENT = 1, /* bad params, null pointers, size mismatch */
    K3DOM_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    K3DOM_ERR_OUT_OF_MEMORY = 3,
    K3DOM_ERR_CAPACITY = 4,         /* a size exceeds a capacity fixed at creation */
    K3DOM_ERR_NOT_READY = 5,        /* call order: e.g. stage before first frame */
    K3DOM_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
    K3DOM_ERR_IO = 7,               /* file could not be read */
    K3DOM_ERR_INVALID_INPUT = 8,    /* non-finite point coordinates */
    K3DOM_ERR_NO_DEVICE = 9
} k3dom_status;

typedef enum k3dom_variant {
    K3DOM_VARIANT_K3DOM = 0,    /* Dirichlet masses + BGKI (src/k3dom) */
    K3DOM_VARIANT_DSPHDMIB = 1  /* Dempster-Shafer masses + inverse sensor model (src/dsphdmib) */
} k3dom_variant;

typedef enum k3dom_mem { K3DOM_MEM_HOST = 0, K3DOM_MEM_DEVICE = 1 } k3dom_mem;

/* Mirrors dom::DOM_c::Params (include/common/dom.h:19-52) field for field, in index
 * units after the node's conversions (k3dom_node.cpp:344-368). The three trailing fields
 * are additions of this library. */
typedef struct k3dom_params {
    float size;
    float size_z;
    float mass_scale;
    float resolution;
    int32_t particle_count;
    int32_t new_born_particle_count;
    float persistence_prob;
    float stddev_process_noise_position;
    float stddev_process_noise_velocity;
    float birth_prob;
    float stddev_velocity;
    float init_max_velocity;
    float particle_min_vel;
    float sensor_off_x;
    float sensor_off_y;
    float sensor_off_z;
    int32_t map_shift_thresh;
    float prior_free;
    float prior_static;
    float prior_dynamic;
    float prior_occ;
    float sigma;           /* K3DOM: sigma_0 of the sparse kernel */
    float ls;              /* K3DOM: kernel length scale [m] */
    float gamma;           /* K3DOM: mass decay per second */
    float max_range;       /* DS-PHD/MIB: inverse sensor model range [m] */
    float meas_occ_stddev; /* DS-PHD/MIB: occupied evidence stddev [m] */
    /* additions */
    uint64_t seed;         /* Philox key of every random draw */
    int32_t max_points;    /* capacity of points per frame (grows on demand, 0 = 131072) */
    int32_t reserved;
} k3dom_params;

typedef struct k3dom_handle k3dom_handle;

/* Node defaults of k3dom_node.cpp:219-258 (K3DOM) or dsphdmib_node.cpp:205-247 (DS),
 * converted to index units exactly as the node does. */
k3dom_status k3dom_params_default(k3dom_variant variant, k3dom_params* out);

/* Reads the flat `key: value` YAML subset of config/<method>.yaml and config/<dataset>.yaml
 * (either path may be NULL), applies them over the node defaults and converts units as
 * k3dom_node.cpp:344-368 / dsphdmib_node.cpp:330-356 do, quirks included (DS reads
 * occupied_thresh into valid_thresh; DS max_range fixed at 50). */
k3dom_status k3dom_params_from_yaml(k3dom_variant variant, const char* method_yaml,
                                    const char* dataset_yaml, k3dom_params* out);

/* Optional: YAML keys that are node-level, not DOM params (thresholds, publishing). */
typedef struct k3dom_node_config {
    float occupied_thresh, valid_thresh, free_thresh, min_z, max_z, min_var, max_var;
    float ds_resolution, imu_pose_offset;
    int32_t map_pub_freq, map_vis_mode, do_eval;
} k3dom_node_config;
k3dom_status k3dom_node_config_from_yaml(k3dom_variant variant, const char* method_yaml,
                                         const char* dataset_yaml, k3dom_node_config* out);

/* DOM_c::DOM_c + DOM::DOM (src/common/dom.cu:29-66, src/k3dom/dom.cu:21-23,
 * src/dsphdmib/dom.cu:21-25). Allocates all device state once on `device`. */
k3dom_status k3dom_create(const k3dom_params* params, k3dom_variant variant, int device,
                          k3dom_handle** out);
k3dom_status k3dom_destroy(k3dom_handle* h);

/* DOM_c::updatePose (src/common/dom.cu:111-158). The map shift runs on the device with no
 * allocation; the particle part of the shift is folded into the next prediction. */
k3dom_status k3dom_update_pose(k3dom_handle* h, float x, float y, float z);

/* The node's cloud transform (k3dom_node.cpp:73-83,99-127: pcl_ros::transformPointCloud of the
 * lidar-frame cloud by tf_lidar2lmap.inverse(), a rotation into the map-aligned frame) done on
 * the GPU: from the next update on, every point p of `scene` (0 for a plain handle) is used as
 * R p + t, with R = rotation (9 floats, row-major) and t = translation (3 floats, NULL = 0),
 * evaluated in FP32 as ((R[0] x + R[1] y) + R[2] z) + t[0] per row without fused multiply-add.
 * rotation = NULL switches the transform off (points as given). Set it before each update whose
 * pose changed; it is part of the frame, so a captured steady frame stays valid. */
k3dom_status k3dom_set_point_transform(k3dom_handle* h, int32_t scene, const float* rotation,
                                       const float* translation);

/* DOM::updateGrid (src/k3dom/dom.cu:29-50, src/dsphdmib/dom.cu:32-53). xs/ys/zs are n
 * point coordinates; ys/zs may be NULL when xs holds n interleaved xyz triples. */
k3dom_status k3dom_update_grid(k3dom_handle* h, float t, const float* xs, const float* ys,
                               const float* zs, int32_t n, k3dom_mem mem);
k3dom_status k3dom_update_grid_async(k3dom_handle* h, float t, const float* xs,
                                     const float* ys, const float* zs, int32_t n,
                                     k3dom_mem mem);
k3dom_status k3dom_synchronize(k3dom_handle* h);
/* The cudaStream_t the handle enqueues on (as void*). */
k3dom_status k3dom_get_stream(k3dom_handle* h, void** stream);
/* Capture the steady-state frame in a CUDA graph (default on). */
k3dom_status k3dom_set_graph_mode(k3dom_handle* h, int enabled);

/* ---- stage calls: the public stage methods of DOM_c / DOM (include/common/dom.h:89-94,
 * include/k3dom/dom.h:23-29, include/dsphdmib/dom.h:23-32). Each runs the same kernels
 * as k3dom_update_grid and synchronises. ---- */
k3dom_status k3dom_particle_prediction(k3dom_handle* h, float dt);
k3dom_status k3dom_particle_assignment(k3dom_handle* h);
/* K3DOM: DOM::gridCellOccupancyUpdate(dt, xs, ys, zs); DS: dt is ignored. */
k3dom_status k3dom_grid_cell_occupancy_update(k3dom_handle* h, float dt, const float* xs,
                                              const float* ys, const float* zs, int32_t n,
                                              k3dom_mem mem);
k3dom_status k3dom_update_persistent_particles(k3dom_handle* h);
k3dom_status k3dom_initialize_new_particles(k3dom_handle* h);
/* Per-cell mean velocities are produced inside the occupancy update; this call exists
 * for call-sequence compatibility and does no GPU work. */
k3dom_status k3dom_statistical_moments(k3dom_handle* h);
k3dom_status k3dom_resampling(k3dom_handle* h);
/* DOM::initializeParticles (first frame, src/k3dom/dom.cu:52-77). */
k3dom_status k3dom_initialize_particles(k3dom_handle* h, const float* xs, const float* ys,
                                        const float* zs, int32_t n, k3dom_mem mem);
/* Copies the resampled set into the persistent set (the deep copy at src/k3dom/dom.cu:43
 * is a buffer flip here) and advances time like updateGrid's tail. */
k3dom_status k3dom_finish_frame(k3dom_handle* h, float t);

/* ---- geometry and scalar getters (include/common/dom.h:59-83) ---- */
typedef struct k3dom_info {
    int32_t grid_size, grid_size_z, grid_cell_count, particle_count,
        new_born_particle_count, iteration, variant, initialized;
    float resolution, center_x, center_y, center_z, sensor_x, sensor_y, sensor_z,
        updated_time;
    int32_t max_points, frame_index;
} k3dom_info;
k3dom_status k3dom_get_info(k3dom_handle* h, k3dom_info* out);
k3dom_status k3dom_index_to_coord(k3dom_handle* h, int32_t idx, float* x, float* y,
                                  float* z);

/* ---- readback (the node's cudaMemcpy of grid_cell_array, k3dom_node.cpp:131-132) ---- */
typedef enum k3dom_cell_field {
    K3DOM_CELL_FREE_MASS = 0,
    K3DOM_CELL_STATIC_MASS = 1,
    K3DOM_CELL_DYNAMIC_MASS = 2,
    K3DOM_CELL_OCC_MASS = 3,
    K3DOM_CELL_PERS_MASS = 4,
    K3DOM_CELL_PRED_MASS = 5,
    K3DOM_CELL_BORN_MASS = 6,
    K3DOM_CELL_MEAN_X_VEL = 7,
    K3DOM_CELL_MEAN_Y_VEL = 8,
    K3DOM_CELL_MEAN_Z_VEL = 9,
    K3DOM_CELL_MU_A = 10,
    K3DOM_CELL_MU_UA = 11,
    K3DOM_CELL_W_A = 12,
    K3DOM_CELL_W_UA = 13,
    K3DOM_CELL_LIKELIHOOD = 14,
    K3DOM_CELL_P_A = 15,
    K3DOM_CELL_OCC_MEAN = 16,   /* GridCell::occ_mean (dom_types.h:48) */
    K3DOM_CELL_DYN_MEAN = 17,   /* GridCell::dyn_mean (dom_types.h:49) */
    K3DOM_CELL_TOTAL_MASS = 18, /* GridCell::total_mass (dom_types.h:47) */
    K3DOM_CELL_OCC_PROB = 19,   /* GridCell::occ_prob (dom_types.h:61) */
    K3DOM_CELL_VAR = 20,        /* GridCell::calcVar (dom_types.h:50-58) */
    K3DOM_CELL_MEAS_OCC = 21,   /* DS: MeasurementCell::occ_mass */
    K3DOM_CELL_MEAS_FREE = 22,  /* DS: MeasurementCell::free_mass */
    K3DOM_CELL_DEL_OCC = 23,    /* K3DOM: last BGKI occupied evidence */
    K3DOM_CELL_DEL_FREE = 24,   /* K3DOM: last BGKI free evidence */
    K3DOM_CELL_FIELD_COUNT = 25
} k3dom_cell_field;
k3dom_status k3dom_get_cell_field(k3dom_handle* h, k3dom_cell_field field, float* dst,
                                  k3dom_mem mem);
/* Registered output (no reference counterpart; the reference's node reads the grid after each
 * updateGrid): from the next frame on, every frame also writes `field` of the selected scene to
 * dst (C floats; device memory, or pinned host memory -- pageable host memory is refused with
 * K3DOM_ERR_INVALID_ARGUMENT). The export runs on a side stream as soon as the field is final
 * and the frame completes only when it has landed, so after k3dom_update_grid returns (or
 * k3dom_synchronize) dst holds the frame's field. dst == NULL stops it. */
k3dom_status k3dom_set_output(k3dom_handle* h, k3dom_cell_field field, float* dst, k3dom_mem mem);
/* start_idx / end_idx per cell (-1 when empty), as particleToGridKernel leaves them. */
k3dom_status k3dom_get_cell_ranges(k3dom_handle* h, int32_t* start, int32_t* end,
                                   k3dom_mem mem);
/* The reference's 68-byte dom::GridCell array (include/common/dom_types.h:12-65). */
#define K3DOM_GRIDCELL_BYTES 68
k3dom_status k3dom_get_gridcell_aos(k3dom_handle* h, void* dst, k3dom_mem mem);
/* The /map_data evaluation cloud of k3dom_node.cpp:161-184: per cell 10 floats
 * x, y, z, v_x, v_y, v_z (m/s), occ_val, dyn_val, eval_aug, dyn_aug (MapPoint,
 * include/common/mappoint.h:5-28, without PCL's padding). */
#define K3DOM_MAPPOINT_FLOATS 10
k3dom_status k3dom_get_mappoints(k3dom_handle* h, float* dst, k3dom_mem mem);

/* Overwrites cell state (masses) -- checkpoint restore and parity tests. Any pointer may
 * be NULL to leave that field alone. */
k3dom_status k3dom_set_cell_masses(k3dom_handle* h, const float* free_mass,
                                   const float* static_mass, const float* dynamic_mass,
                                   const float* occ_mass, k3dom_mem mem);

/* ---- particles (ParticlesSoA, include/common/dom_types.h:76-167) ---- */
typedef enum k3dom_particle_set {
    K3DOM_PARTICLES_PERSISTENT = 0, /* particle_array (current) */
    K3DOM_PARTICLES_SORTED = 1,     /* particle_array after assignment (sorted by cell) */
    K3DOM_PARTICLES_BIRTH = 2       /* birth_particle_array */
} k3dom_particle_set;
/* Any output may be NULL. pos/vel are n*3 interleaved floats. */
k3dom_status k3dom_get_particles(k3dom_handle* h, k3dom_particle_set set, float* pos,
                                 float* vel, float* weight, int32_t* cell_idx,
                                 uint8_t* associated, k3dom_mem mem);
k3dom_status k3dom_set_particles(k3dom_handle* h, k3dom_particle_set set, const float* pos,
                                 const float* vel, const float* weight,
                                 const int32_t* cell_idx, const uint8_t* associated,
                                 k3dom_mem mem);
/* Debug / parity hooks. */
/* The permutation of the last assignment: sorted slot i holds the particle that was at
 * index perm[i] before the sort. */
k3dom_status k3dom_get_sort_permutation(k3dom_handle* h, int32_t* perm, k3dom_mem mem);
/* Ancestor index of every resampled particle (0..P+B-1; >= P means birth slot - P). */
k3dom_status k3dom_get_ancestors(k3dom_handle* h, int32_t* anc, k3dom_mem mem);
/* Joint cumulative weights (P+B floats), born-mass cumulative (C floats), joint max. */
k3dom_status k3dom_get_resampling_state(k3dom_handle* h, float* joint_cum,
                                        float* born_cum, float* joint_max, k3dom_mem mem);
/* The draws the library uses: stage 1 = prediction normals (6 per item), 2 = first-frame
 * velocities (3 uniforms, (0,1]), 3 = birth velocities (3 uniforms), 4 = resampling (1
 * uniform). Writes count*per_item floats for items [first, first+count) of frame `frame`. */
k3dom_status k3dom_debug_draws(uint64_t seed, int32_t frame, int32_t stage, int64_t first,
                               int64_t count, float* dst, k3dom_mem mem);
/* The particle sort's bounded waits (test hook; no counterpart in the reference). Each pass of
 * the sort finds the keys of earlier tiles by polling their published counts; a poll loop gives
 * up after max_polls polls (default 1,048,576, under a second), and the frame then returns
 * K3DOM_ERR_TIMEOUT (its results are incomplete). skip_tile >= 0 keeps that tile of the first
 * pass from publishing its counts, so every later tile's wait runs out: how the tests see the
 * timeout path without a hang. skip_tile = -1 restores normal operation. */
k3dom_status k3dom_set_sort_wait(k3dom_handle* h, uint32_t max_polls, int32_t skip_tile);
/* Sets the frame counter used to key the draws (tests align it with a reference run). */
k3dom_status k3dom_set_frame_index(k3dom_handle* h, int32_t frame);

/* Per-stage device time of the last frame in milliseconds (CUDA events). */
typedef struct k3dom_stage_times {
    float predict_ms, assign_ms, occupancy_ms, persistent_ms, births_ms, resample_ms,
        total_ms;
    float binning_ms;  /* part of occupancy_ms: ray lists */
    float evidence_ms; /* part of occupancy_ms: evidence + cell update kernel(s) */
} k3dom_stage_times;
k3dom_status k3dom_get_stage_times(k3dom_handle* h, k3dom_stage_times* out);
k3dom_status k3dom_set_timing(k3dom_handle* h, int enabled);

/* Diagnostics collected on the device for the last frame: points skipped as non-finite (device
 * scans; host scans with such points are refused), ray-list use, work items, evaluations. */
typedef struct k3dom_diagnostics {
    int64_t nonfinite_points, ray_list_entries, ray_list_capacity, work_items;
    int32_t overflow;
    int32_t kernel_launches_per_frame; /* kernels a steady-state frame enqueues (with its point upload) */
    int64_t kernel_evaluations;        /* K3DOM: in-support sparse-kernel evaluations, last frame */
} k3dom_diagnostics;
k3dom_status k3dom_get_diagnostics(k3dom_handle* h, k3dom_diagnostics* out);

/* ---- batches: S independent scenes updated together, one launch per stage ----
 * No counterpart in the reference, whose DOM holds one scene. Each scene keeps its own
 * parameters, pose, clock and draw stream, and a scene updated in a batch produces exactly the
 * results of the same scene in a handle of its own. A plain handle is a batch of one; the
 * per-scene getters and setters above (info, cell fields, ranges, GridCell / MapPoint export,
 * particles, permutation, ancestors, resampling state, cell masses, update_pose) address the
 * scene chosen with k3dom_select_scene (scene 0 by default). At most 64 scenes. */
k3dom_status k3dom_batch_create(const k3dom_params* params, int32_t n_scenes, k3dom_variant variant,
                                int device, k3dom_handle** out);
k3dom_status k3dom_batch_size(k3dom_handle* h, int32_t* n_scenes);
k3dom_status k3dom_select_scene(k3dom_handle* h, int32_t scene);
k3dom_status k3dom_batch_update_pose(k3dom_handle* h, int32_t scene, float x, float y, float z);
/* One frame of every scene: scene s gets time t[s] and points xs[s], ys[s], zs[s] (n[s] of
 * them; ys/zs may be NULL, or ys[s]/zs[s] NULL, for interleaved xyz in xs[s]). All scenes are
 * in the same phase: the first call initialises every scene. */
k3dom_status k3dom_batch_update(k3dom_handle* h, const float* t, const float* const* xs,
                                const float* const* ys, const float* const* zs, const int32_t* n,
                                k3dom_mem mem);
k3dom_status k3dom_batch_update_async(k3dom_handle* h, const float* t, const float* const* xs,
                                      const float* const* ys, const float* const* zs,
                                      const int32_t* n, k3dom_mem mem);

/* ---- evidence tuning ----
 * The evidence stage's tile shape (rule 0: 16x16x8 cells for grids of >= 2^20 cells, else
 * 8x8x4; 1: 8x8x4; 2: 16x16x4; 3: 16x16x8) and rays per work item (chunk) change its speed,
 * never its results. k3dom_autotune(h, 1) measures every (rule, chunk in {512, 1024})
 * candidate on the next steady frames, one candidate per frame (those frames are run without
 * the graph), then keeps the fastest. candidate_ms[k] belongs to rule k % 4 with chunk
 * {512, 1024}[k / 4]. */
#define K3DOM_TUNE_MAX_CANDIDATES 16
typedef struct k3dom_tuning {
    int32_t tile_rule, chunk, tuned, tuning, candidates, evidence_blocks;
    float best_ms;
    float candidate_ms[K3DOM_TUNE_MAX_CANDIDATES]; /* evidence stage time of each candidate */
    /* evidence_blocks: CTAs of the K3DOM evidence launch, or of the DS final (update) pass;
     * evidence_count_blocks: CTAs of the DS count pass (0 for K3DOM). Both grids are
     * persistent, one CTA per resident slot of the build that runs. */
    int32_t evidence_count_blocks;
} k3dom_tuning;
k3dom_status k3dom_autotune(k3dom_handle* h, int enabled);
k3dom_status k3dom_get_tuning(k3dom_handle* h, k3dom_tuning* out);
k3dom_status k3dom_set_tuning(k3dom_handle* h, int32_t tile_rule, int32_t chunk);

/* ---- the differentiable kernel-inference update (calibration) ----
 * No counterpart in the reference. A calibration problem holds a grid (from `base`), training
 * frames (points, sensor pose, dt; frame 0 initialises with dt = 0, later frames may carry the
 * particle weight sum of every cell, which is treated as data: sort and resampling are not
 * differentiated) and held-out scans, whose rays are traversed by 3-D DDA into per-cell label
 * counts (hit voxel: label 1; voxels traversed before it: label 0).
 * theta[5] = { kernel length-scale ls [m], kernel amplitude sigma, free-space decay gamma
 * (pred_total = (free + dynamic) * gamma^dt, mass_update.cu:166), occupied prior mass (split
 * evenly into the static and dynamic priors), free prior mass }.
 * Loss = mean binary cross-entropy between the occupancy (static + dynamic) / total after the
 * last frame (clamped to [1e-7, 1 - 1e-7]) and the labels, over all label instances.
 * Points are sensor-relative xyz triples (n x 3, interleaved); the sensor position is relative
 * to the grid centre. */
typedef struct k3dom_calib k3dom_calib;
k3dom_status k3dom_calib_create(const k3dom_params* base, int device, k3dom_calib** out);
k3dom_status k3dom_calib_destroy(k3dom_calib* c);
/* dyn_pred: grid_cell_count floats (NULL: no particles); ignored for frame 0. */
k3dom_status k3dom_calib_add_frame(k3dom_calib* c, float dt, float sensor_x, float sensor_y,
                                   float sensor_z, const float* xyz, int32_t n,
                                   const float* dyn_pred, k3dom_mem mem);
k3dom_status k3dom_calib_add_heldout_scan(k3dom_calib* c, float sensor_x, float sensor_y,
                                          float sensor_z, const float* xyz, int32_t n,
                                          k3dom_mem mem);
k3dom_status k3dom_calib_label_counts(k3dom_calib* c, uint32_t* n0, uint32_t* n1, k3dom_mem mem);
/* Per-cell sums of frame `frame` at length-scale ls: 4 x grid_cell_count doubles
 * (sum f occupied, sum f free, sum -x f'(x) occupied, sum -x f'(x) free; x = d / ls). */
k3dom_status k3dom_calib_get_sums(k3dom_calib* c, float ls, int32_t frame, double* out, k3dom_mem mem);
k3dom_status k3dom_calib_info(k3dom_calib* c, int32_t* cells, int32_t* frames,
                              double* label_instances);
k3dom_status k3dom_calib_get_stream(k3dom_calib* c, void** stream);
/* Loss at theta; occupancy (grid_cell_count floats, may be NULL) receives p(c). */
k3dom_status k3dom_bgki_forward(k3dom_calib* c, const float* theta, float* loss, float* occupancy,
                                k3dom_mem mem);
/* grad_theta[i] = grad_loss * dLoss/dtheta[i] by the hand-written adjoint; loss may be NULL. */
k3dom_status k3dom_bgki_backward(k3dom_calib* c, const float* theta, float grad_loss,
                                 float* grad_theta, float* loss);

/* Exact inclusive prefix sum of n non-negative floats (device pointers in/out, enqueued on
 * `stream`, a cudaStream_t or NULL) that allocates no memory: its scratch is a fixed 256 KiB
 * array inside the library on each GPU. For callers that may not allocate device memory at
 * run time. The sum is the one the update uses for birth slots and ancestors: each prefix is
 * the correctly rounded exact sum, for finite inputs in [0, 2^23) (-0 counts as 0; inputs
 * below 2^-56 enter truncated to a multiple of 2^-80). Any other element (negative, NaN,
 * infinite, >= 2^23) is refused on the device: out[i] is NaN from the first such element on
 * (the call does not synchronise, so this cannot be a status). n <= 33,554,432 (else
 * K3DOM_ERR_CAPACITY, nothing enqueued). Calls share the scratch: calls that overlap on the GPU
 * race. The first call in each CUDA context looks up the scratch address; make it before any
 * stream capture. Its launches are not counted in any handle's launch figures, and a launch
 * failure returns K3DOM_ERR_CUDA without consuming an unrelated earlier CUDA error. No
 * counterpart in the reference. */
k3dom_status k3dom_exact_prefix_sum_noalloc(const float* in, float* out, int64_t n, void* stream);

const char* k3dom_status_string(k3dom_status s);
/* The CUDA runtime's message for the last CUDA error a call on this handle met
 * ("no error" when none). */
const char* k3dom_last_cuda_error(k3dom_handle* h);
int32_t k3dom_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* K3DOM_B200_H */
