/*
 * cublox_b200 — C ABI of the B200 (sm_100a) map-integration path.
 *
 * Plain C types only.  Every call returns CUBLOX_OK (0) or a negative status;
 * cublox_last_error() gives the message of the calling thread's last failure.
 * Citations name the reference interface (mrsp/cublox) each entry replaces.
 *
 * Streams: every grid owns (or borrows) one CUDA stream; all of its device
 * work is ordered on it.  Calls that return host data wait for that stream;
 * cublox_grid_update* only enqueue (the host cloud is staged into pinned
 * memory before the call returns, so the caller may reuse its buffer).
 */
#ifndef CUBLOX_B200_H
#define CUBLOX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUBLOX_OK 0
#define CUBLOX_ERR_INVALID -1 /* bad argument                              */
#define CUBLOX_ERR_CUDA -2    /* CUDA runtime error (message has details) */
#define CUBLOX_ERR_NOMEM -3   /* device or pinned allocation failed       */
#define CUBLOX_ERR_RANGE -4   /* voxel count above int32 (Grid.cpp:44-50) */
#define CUBLOX_ERR_DEVICE -5  /* device-side check failed (error word)    */
#define CUBLOX_ERR_CANCELLED -6 /* served request withdrawn before it ran  */

#define CUBLOX_STATE_UNKNOWN 0 /* OccupancyGrid.hpp:31-35 */
#define CUBLOX_STATE_FREE 1
#define CUBLOX_STATE_OCCUPIED 2
#define CUBLOX_FILTER_ALL (-1)

/* Point-cloud layouts accepted by cublox_grid_update_xyz.                   */
#define CUBLOX_LAYOUT_SOA 0 /* x[0..n), y[0..n), z[0..n) back to back       */
#define CUBLOX_LAYOUT_AOS 1 /* x0 y0 z0 x1 y1 z1 ...                        */

typedef struct cublox_grid cublox_grid;

/* Per-scan algorithmic counters (filled when stats are enabled).            */
typedef struct {
  int64_t rays;        /* points not dropped (finite, length >= 1e-6)      */
  int64_t op_incs;     /* in-window op increments incl. endpoints (U)      */
  int64_t hit_incs;    /* endpoint hits (H)                                 */
  int64_t touched;     /* voxels whose counters were folded (T)            */
} cublox_scan_stats;

const char *cublox_last_error(void);
const char *cublox_version(void);
/* Binary version of this library's kernels as loaded on the current device
 * (major * 10 + minor: 100 for sm_100a).  No counterpart in the reference.  */
int cublox_binary_version(int *binary_version);
/* Process-wide counts of what this library has done so far, for checking
 * that a steady state allocates nothing: out[0] device allocations, [1]
 * device frees, [2] pinned host allocations, [3] pinned host frees, [4] CUDA
 * graphs instantiated.  Fills the first n (entries past 5 read 0).  No
 * counterpart in the reference.                                             */
int cublox_runtime_counters(int64_t *out, int n);
/* Test hook: once `skip` more device or pinned allocations have been made,
 * the next `count` fail as if memory were exhausted (no CUDA call is made;
 * the failing call returns CUBLOX_ERR_NOMEM or its caller's error), so that
 * tests can drive the out-of-memory paths without exhausting a GPU; count 0
 * turns it off.  Process-wide.  No counterpart in the reference, whose
 * CUDA_OK aborts the process on any failed call (OccupancyGrid.cpp:32-49). */
int cublox_test_fail_allocations(int64_t skip, int64_t count);
/* Measures the device's throughput of 32-bit atomic adds whose result is
 * unused (the walk's only memory operation) to pseudo-random distinct
 * addresses of a buffer of buffer_bytes (allocated and freed by the call):
 * about total_ops operations, timed with CUDA events on `stream`.  The
 * denominator of the walk's L2-atomic roofline.  No counterpart in the
 * reference.                                                                */
int cublox_probe_red_rate(int64_t buffer_bytes, int64_t total_ops, void *stream,
                          double *ops_per_s);

/* OccupancyGrid(half_map_size_i, resolution, origin_at_center,
 * recenter_threshold, origin)  — OccupancyGrid.hpp:42-45,
 * OccupancyGrid.cpp:54-65, Grid.cpp:27-54.  `stream` is a cudaStream_t or
 * NULL (the grid then creates its own non-blocking stream).                 */
int cublox_grid_create(const int half_map_size[3], float resolution,
                       int origin_at_center, int has_recenter_threshold,
                       double recenter_threshold, const float origin[3],
                       void *stream, cublox_grid **out);
/* ~OccupancyGrid — OccupancyGrid.cpp:67-114.                               */
int cublox_grid_destroy(cublox_grid *g);

/* reset() / resetVoxel(hash) — OccupancyGrid.cpp:116-139.                  */
int cublox_grid_reset(cublox_grid *g);
int cublox_grid_reset_voxel(cublox_grid *g, int hash_id);

/* setMaxRaycastRange / getMaxRaycastRange — OccupancyGrid.hpp:68-71.       */
int cublox_grid_set_max_range(cublox_grid *g, float range);
int cublox_grid_get_max_range(const cublox_grid *g, float *range);
/* setLogOddsParams — OccupancyGrid.hpp:74-85 (l_unknown stays 0).         */
int cublox_grid_set_log_odds(cublox_grid *g, float l_hit, float l_miss,
                             float l_min, float l_max, float l_free,
                             float l_occupied);

/* FP32 multiply-add contraction pattern to reproduce.  Bits 0-2: shape of
 * the ray-length sum of squares (0 plain, 1 fma(z,z,fma(y,y,x*x)),
 * 2 fma(z,z,fma(x,x,y*y)), 3 fma(z,z,x*x+y*y), 4 fma(y,y,x*x)+z*z,
 * 5 fma(x,x,y*y)+z*z); bit 3 clip point; bit 4 voxel-boundary distance;
 * bit 5 centre binning; bits 6/7 miss/hit log-odds terms; bits 8-10 and
 * 11-13 the recenter-gate and fetch sums of squares; bit 14 fetch offset.
 * The default is the pattern of the reference's own sm_100a release build,
 * pinned black-box by tests/test_contraction_pins.py.                      */
int cublox_grid_set_fp_mode(cublox_grid *g, unsigned mode);
int cublox_grid_get_fp_mode(const cublox_grid *g, unsigned *mode);

/* Kernel choices (no reference counterpart; results are identical for
 * every choice, only speed differs).                                       */
#define CUBLOX_OPT_RAYCAST 1 /* 0: one thread per ray; 1: direction-binned
                                warp walk; 2: rays split between lanes at
                                exact time cuts (default)                  */
#define CUBLOX_OPT_CUBE 2    /* shared-memory counter cube side around the
                                sensor: 0, 8, 16 or 32 (default 32; 8 is
                                split walk only)                           */
#define CUBLOX_OPT_MATCH 3   /* merge duplicate voxels per warp (default 0) */
#define CUBLOX_OPT_SORT 4    /* walk rays in direction order (default 0)    */
#define CUBLOX_OPT_SEGMENT 5 /* split walk: in-window steps per lane (64)   */
#define CUBLOX_OPT_FOLD 6    /* fold: 0 scalar sweep of every counter, 1
                                16-byte sweep; only the 32-voxel lines the
                                scan flagged: 2 (default) compacted into a
                                list per 4096 lines, 3 read 32 flags at a
                                time per warp                              */
#define CUBLOX_OPT_BLOCK 7   /* split walk CTA size: 256, 512, 1024         */
#define CUBLOX_OPT_CONTIGUOUS 8 /* split walk: each CTA walks one run of
                                   consecutive segments (default 0: all
                                   CTAs share one segment queue)            */
#define CUBLOX_OPT_FLAT_CUBE 10 /* split walk with cube 32: a 32 x 32 x 16
                                   cube (half the height, two CTAs per SM);
                                   0 (default) or 1                      */
#define CUBLOX_OPT_LAYOUT 9  /* voxel layout of the grid's arrays: log2 of
                                the brick sides as decimal digits x y z,
                                bricks of 32 voxels (320: 8 x 4 x 1, the
                                default; 230; 221), or 0 for the
                                reference's hash order.  Setting it moves
                                the stored map (between scans).  Every
                                layout gives identical results; exports
                                and hash arguments always use the
                                reference's hash order.                    */
int cublox_grid_set_option(cublox_grid *g, int key, int value);
int cublox_grid_get_option(const cublox_grid *g, int key, int *value);

/* update(cloud, sensor_origin) — OccupancyGrid.hpp:53-54,
 * OccupancyGrid.cpp:181-238.  x/y/z are the three columns of the reference's
 * column-major PointCloud (host or device pointers; n points each).         */
int cublox_grid_update(cublox_grid *g, const float *x, const float *y,
                       const float *z, int n, const float sensor_origin[3]);
/* Same, with the cloud in one buffer of the given layout.                   */
int cublox_grid_update_xyz(cublox_grid *g, const float *xyz, int layout,
                           int n, const float sensor_origin[3]);
/* update() from a sensor-frame cloud and the sensor's pose: what the
 * reference's driver does before calling update() (buildCloudInOdomFrame,
 * src/main.cpp:640-693, called at :450-452) — drop non-finite points and
 * points farther than the max raycast range, map the rest to the world as
 * rotation * p + translation (rotation row-major) — done on the device,
 * followed by update(world_cloud, translation).  A cloud with no point left
 * leaves the grid untouched, as the driver then skips update().             */
int cublox_grid_update_pose(cublox_grid *g, const float *xyz, int layout, int n,
                            const float rotation[9], const float translation[3]);

/* Depth image encodings of cublox_grid_update_depth (depthCallback,
 * src/main.cpp:572-573).                                                    */
#define CUBLOX_DEPTH_U16_MM 0 /* 16UC1 / mono16: millimetres, 0 = no return  */
#define CUBLOX_DEPTH_F32_M 1  /* 32FC1: metres, non-finite or <= 0 = none    */
/* update() from a depth image (height rows of `step` bytes, host or device):
 * the reference driver's depthCallback (src/main.cpp:558-638) makes one
 * camera-frame point per pixel, x = ((u - cx) * z) / fx, y = ((v - cy) * z)
 * / fy, then the cloud goes through cublox_grid_update_pose.  intrinsics =
 * {fx, fy, cx, cy} (K(0,0), K(1,1), K(0,2), K(1,2)).                        */
int cublox_grid_update_depth(cublox_grid *g, const void *image, int encoding, int width,
                             int height, int64_t step, const float intrinsics[4],
                             const float rotation[9], const float translation[3]);

/* recenter(pos) — OccupancyGrid.hpp:57, OccupancyGrid.cpp:141-179.
 * *action (may be NULL): 0 nothing, 1 slabs cleared, 2 full reset.
 * mode 0 reproduces the reference's slab set exactly (its extra band of
 * "entering" slabs included); mode 1 clears only the slabs that left.      */
int cublox_grid_recenter(cublox_grid *g, const float pos[3], int *action);
int cublox_grid_set_recenter_mode(cublox_grid *g, int mode);

/* fetchOccupancyAround(center, radius, filter, max_results) —
 * OccupancyGrid.hpp:62-65, OccupancyGrid.cpp:240-356.  filter is -1 (all)
 * or a CUBLOX_STATE_*.  Samples come in ascending (x, y, z) global-index
 * order; out_pos holds 3 floats per sample.  Writes at most `capacity`;
 * *n_out = samples returned (as the reference returns them).               */
int cublox_grid_fetch(cublox_grid *g, const float center[3], float radius,
                      int filter, int max_results, float *out_pos,
                      uint8_t *out_state, int64_t capacity, int64_t *n_out);
/* The driver's visualisation cloud (src/main.cpp:740-790) of one fetch:
 * the samples in fetch order, dropped unless (gx ^ gy ^ gz) % subsample_step
 * == 0 for their global index (:71-84), coloured by distance to robot_pos
 * over max_viz_radius (:275-289) and packed as x, y, z, rgb floats (the rgb
 * float carries 0x00RRGGBB, :291-302); at most max_points.  Built on the
 * device from the fetch's samples; *n_out gets the points written.       */
int cublox_grid_fetch_viz(cublox_grid *g, const float center[3], float radius, int filter,
                          int max_results, int subsample_step, float max_viz_radius,
                          int64_t max_points, const float robot_pos[3], float *out_xyzrgb,
                          int64_t capacity, int64_t *n_out);

/* Many fetches in one launch (no reference counterpart beyond calling
 * fetchOccupancyAround once per centre).  out_offsets gets n_centers+1
 * entries; query q's samples are [out_offsets[q], out_offsets[q+1]).
 * Output buffers are host pointers.  If capacity is too small the call
 * fills out_offsets and returns CUBLOX_ERR_INVALID without samples.       */
int cublox_grid_fetch_batch(cublox_grid *g, const float *centers,
                            int n_centers, float radius, int filter,
                            int max_results, int64_t *out_offsets,
                            float *out_pos, uint8_t *out_state,
                            int64_t capacity);
/* Counts only: per-centre sample counts, no samples materialised.         */
int cublox_grid_fetch_counts(cublox_grid *g, const float *centers,
                             int n_centers, float radius, int filter,
                             int max_results, int64_t *out_counts);

/* isOccupied/isFree/isUnknown(pos) — OccupancyGrid.cpp:368-393, for n
 * points in one launch: out_state[i] = CUBLOX_STATE_* of point i (outside
 * the window: UNKNOWN).                                                     */
int cublox_grid_query_states(cublox_grid *g, const float *xyz, int n,
                             uint8_t *out_state);
/* storedAt(hash) — OccupancyGrid.cpp:358-366 (0 for an out-of-range hash). */
int cublox_grid_stored_at(cublox_grid *g, int hash_id, float *out);

/* getOriginIndex / getOriginPosition — Grid.hpp:37-38.                    */
int cublox_grid_origin(const cublox_grid *g, int origin_i[3],
                       float origin_f[3]);
/* Grid::Config — Grid.hpp:44-53.                                           */
int cublox_grid_geometry(const cublox_grid *g, int map_size[3], int half[3],
                         int *voxel_num, float *resolution,
                         int *origin_at_center);
/* first_run_ flag of the reference (OccupancyGrid.cpp:192-198): 1 until the
 * first update snaps the window origin to the sensor.                      */
int cublox_grid_first_run(const cublox_grid *g, int *first_run);
/* Force the window origin (global voxel index); clears first_run.          */
int cublox_grid_set_origin_index(cublox_grid *g, const int origin_i[3]);

/* The stored log-odds of every voxel, in the reference's ring-buffer hash
 * order (utils.cuh:131-136), into a host buffer of voxel_num floats.       */
int cublox_grid_export(cublox_grid *g, float *occ_host);
int cublox_grid_import(cublox_grid *g, const float *occ_host);

/* Stream handling.                                                          */
int cublox_grid_stream(const cublox_grid *g, void **stream);
int cublox_grid_synchronize(cublox_grid *g);

/* Algorithmic counters of the last update (enable first; costs one extra
 * device->host copy per update when read).                                 */
int cublox_grid_enable_stats(cublox_grid *g, int enable);
int cublox_grid_last_stats(cublox_grid *g, cublox_scan_stats *out);

/* Raycast one scan (AoS host points) without folding it, return the per-
 * voxel traversal and hit counts the reference keeps in op_cnt / hit_cnt
 * (kernels.cu:33-152; ring-buffer hash order), then zero them.  The map is
 * left unchanged.  For verification.                                       */
int cublox_grid_count_scan(cublox_grid *g, const float *xyz, int n,
                           const float sensor_origin[3], int32_t *op_out,
                           int32_t *hit_out);

/* Device time of the last raycast, fold and recenter-clear launches in ms
 * (-1 where none ran since the last read); timing is opt-in.               */
int cublox_grid_enable_timing(cublox_grid *g, int enable);
int cublox_grid_last_timing(cublox_grid *g, float ms[3]);
/* Voxels the last recenter cleared (its slab union, or every voxel on a
 * full reset; 0 when it did nothing).  Accounting only, no reference
 * counterpart.                                                              */
int cublox_grid_last_clear(const cublox_grid *g, int64_t *voxels);

/* Work units of one scan as the reference counts them: per ray, the DDA
 * iterations of rayCastUpdateKernel's loop that did not break, plus one for
 * the endpoint (kernels.cu:105-151), over the current window.  Accounting
 * only; no map state changes.                                              */
int cublox_grid_reference_steps(cublox_grid *g, const float *xyz, int n,
                                const float sensor_origin[3],
                                int64_t *voxel_steps);

/* Device error word: nonzero if a kernel's own bounds checks rejected an
 * index (a bug, never expected), or a fused batch launch stopped waiting
 * for the map's walk and skipped its fold (CUBLOX_DEVICE_WAIT_TIMEOUT).
 * Reading it clears it.                                                     */
#define CUBLOX_DEVICE_HASH_RANGE (1u << 0)
#define CUBLOX_DEVICE_FETCH_OVERFLOW (1u << 1)
#define CUBLOX_DEVICE_JUMP_STALL (1u << 2)
#define CUBLOX_DEVICE_WAIT_TIMEOUT (1u << 3)
int cublox_grid_check(cublox_grid *g, uint32_t *error_word);

/* ---- batched integration ----------------------------------------------------
 * No single counterpart in the reference, whose caller integrates one map's
 * scan at a time (OccupancyGrid::update per map).  A batch owns grids created
 * through it (they share its stream and stay usable through every
 * cublox_grid_* call) and integrates one scan into each of many of them in
 * one persistent walk launch and one fold launch, or (fused shapes) in one
 * persistent launch that folds each map as soon as its walk is done.
 * Results are identical to calling cublox_grid_update on each grid.         */
typedef struct cublox_batch cublox_batch;

#define CUBLOX_BATCH_OPT_GRAPHS 1     /* replay the launch sequence from a CUDA
                                         graph (default 0)                  */
#define CUBLOX_BATCH_OPT_AUTOTUNE 2   /* choose the launch shape and the
                                         voxel layout over the first
                                         updates (default 1): each candidate
                                         (every shape with 8 x 4 x 1
                                         bricks, the flat-cube shape with
                                         the other layouts) is timed twice  */
#define CUBLOX_BATCH_OPT_SHAPE 3      /* fix the launch shape (0 .. n-1)    */
#define CUBLOX_BATCH_OPT_TIMING 4     /* record walk/fold device times      */
#define CUBLOX_BATCH_OPT_NUM_SHAPES 5 /* read only: number of shapes        */
#define CUBLOX_BATCH_OPT_FOLD 6       /* fold: 0 (default) the 32-voxel
                                         lines the walk flagged, compacted
                                         into a list per 2048 lines; 1 every
                                         line (the reference's full sweep,
                                         for comparison); 2 the flagged
                                         lines, 32 flags at a time per
                                         warp                               */
#define CUBLOX_BATCH_OPT_LAYOUT 8     /* voxel layout the batch keeps its
                                         grids in (CUBLOX_OPT_LAYOUT codes;
                                         default 320); setting it stops
                                         the tuner                          */
#define CUBLOX_BATCH_OPT_WAIT_LIMIT 9 /* fused shapes: rounds of a ~256 ns
                                         sleep a map's fold waits for its
                                         walk before it gives up, flags
                                         CUBLOX_DEVICE_WAIT_TIMEOUT in the
                                         map's error word and lets the
                                         launch finish without folding
                                         (default 1 << 23, about 2 s)       */
#define CUBLOX_BATCH_OPT_INJECT_MISSING_WALK 10 /* test hook: with a fused
                                         shape, the first map's folds wait
                                         for a walk item that does not
                                         exist, so the wait runs out; the
                                         maps are then left unfolded and
                                         must be reset                      */
#define CUBLOX_BATCH_OPT_HOST_READ 11 /* host points (pinned, or staged in
                                         the batch's pinned buffer): 1
                                         (default) the walk reads them in
                                         place over the bus, each point once,
                                         while it runs; 0 copy them to the
                                         device before the walk             */
#define CUBLOX_BATCH_OPT_TUNING 7     /* read only: 1 while the tuner is
                                         still timing candidate shapes (the
                                         updates until it reads 0 run
                                         shapes other than the best, each
                                         synchronised to be timed)          */

int cublox_batch_create(void *stream, cublox_batch **out);
int cublox_batch_destroy(cublox_batch *b);
/* A grid integrated by this batch (same arguments as cublox_grid_create).   */
int cublox_batch_add_grid(cublox_batch *b, const int half_map_size[3], float resolution,
                          int origin_at_center, int has_recenter_threshold,
                          double recenter_threshold, const float origin[3],
                          cublox_grid **out);
int cublox_batch_set_option(cublox_batch *b, int key, int value);
int cublox_batch_get_option(const cublox_batch *b, int key, int *value);
/* One scan into each of grids[0..n): scan i is points [offsets[i],
 * offsets[i+1]) of xyz (x0 y0 z0 x1 ..., host or device) from sensor
 * origin sensors[3i..3i+2].  A grid may appear once per call.               */
int cublox_batch_update(cublox_batch *b, int n, cublox_grid *const *grids, const float *xyz,
                        const int64_t *offsets, const float *sensors);
/* recenter(pos) of each grid (OccupancyGrid.cpp:141-179); actions may be
 * NULL.                                                                      */
int cublox_batch_recenter(cublox_batch *b, int n, cublox_grid *const *grids,
                          const float *positions, int *actions);
/* Size the batch's buffers for updates of up to `points` points over `maps`
 * grids now, so that later updates of that size allocate nothing (growing
 * a buffer frees the old one, which waits for the whole device).           */
int cublox_batch_reserve(cublox_batch *b, int64_t points, int maps);
/* The same for updates over up to `maps` grids of `voxels` voxels in all,
 * whatever their sizes (the fold's work items grow with the voxels).       */
int cublox_batch_reserve_maps(cublox_batch *b, int64_t points, int maps, int64_t voxels);
int cublox_batch_synchronize(cublox_batch *b);
int cublox_batch_last_timing(cublox_batch *b, float *walk_ms, float *fold_ms);
int cublox_batch_stream(const cublox_batch *b, void **stream);

/* ---- served integration -----------------------------------------------------
 * No single counterpart in the reference, whose ROS driver serialises one
 * robot's callbacks on one grid (main.cpp:464-491).  A server keeps many
 * robots' maps and serves their scan and fetch requests from a worker
 * thread: requests are copied and queued at submission; each "tick"
 * integrates the oldest pending scan of every map that has one (up to
 * max_tick_points) in one batched launch sequence, the next tick being
 * queued while the previous one still runs.  Maps are admitted to device
 * memory against hbm_budget_bytes (12 B a voxel, the tick's point buffers
 * and the fetch buffers maps keep between requests; a fetch in flight may
 * exceed it by its own output buffers until it ends): when a map's
 * buffers do not fit, least recently used idle maps are evicted to host
 * memory and restored bit for bit when next used.  Per map, requests take
 * effect in submission order, and every result equals that of the same
 * requests on a lone cublox_grid.                                           */
typedef struct cublox_server cublox_server;

typedef struct cublox_server_config {
  uint64_t hbm_budget_bytes; /* device bytes for resident maps + scratch     */
  int max_tick_points;       /* points per batched launch (0: 1 << 20)       */
  int max_tick_maps;         /* scans per batched launch (0: no limit)       */
  int max_inflight_ticks;    /* ticks queued on the device (0: 2)            */
  int graphs;                /* replay batched launches from CUDA graphs     */
  /* Everything below is sized when the server is created, so that serving
   * within these sizes allocates nothing (cublox_runtime_counters).        */
  uint64_t pinned_pool_bytes; /* pinned host arena that submitted scans are
                                 copied into (0: 256 MiB); a scan that finds
                                 no room stays in pageable memory           */
  int max_fetch_centres;      /* centres per fetch request (0: 1024)        */
  int64_t max_fetch_samples;  /* samples per fetch request (0: 1 << 22)     */
} cublox_server_config;

typedef struct cublox_server_stats {
  int64_t ticks, scans, fetches, points; /* served so far                  */
  int64_t admissions, evictions;         /* maps brought in / sent to host */
  uint64_t resident_bytes, peak_resident_bytes;
  int resident_maps;
  int64_t cancelled;                     /* requests withdrawn             */
} cublox_server_stats;

#define CUBLOX_REQ_QUEUED 0
#define CUBLOX_REQ_RUNNING 1
#define CUBLOX_REQ_DONE 2
#define CUBLOX_REQ_FAILED 3

int cublox_server_create(const cublox_server_config *cfg, cublox_server **out);
int cublox_server_destroy(cublox_server *s);
/* A robot's map: the OccupancyGrid constructor's arguments, its max raycast
 * range and log-odds (setLogOddsParams order; NULL keeps the defaults).     */
int cublox_server_add_map(cublox_server *s, const int half_map_size[3], float resolution,
                          int origin_at_center, int has_recenter_threshold,
                          double recenter_threshold, const float origin[3], float max_range,
                          const float log_odds[6], int *map_id);
/* update(cloud, sensor_origin) (OccupancyGrid.cpp:181-238) on the map, then
 * recenter(sensor_origin) if `recenter`; xyz is x0 y0 z0 x1 ... on the host,
 * copied before the call returns (into the server's pinned pool, up to
 * 1 GiB, else pageable memory).                                             */
int cublox_server_submit_scan(cublox_server *s, int map_id, const float *xyz, int n,
                              const float sensor_origin[3], int recenter,
                              int64_t *request_id);
/* fetchOccupancyAround for each centre (OccupancyGrid.cpp:240-356).         */
int cublox_server_submit_fetch(cublox_server *s, int map_id, const float *centers,
                               int n_centers, float radius, int filter, int max_results,
                               int64_t *request_id);
/* Wait until the request is done or failed (timeout_s < 0: no limit); state
 * gets CUBLOX_REQ_*.  A failed request returns its error.                   */
int cublox_server_wait(cublox_server *s, int64_t request_id, double timeout_s, int *state);
int cublox_server_drain(cublox_server *s); /* every submitted request done  */
/* Submission-to-start and submission-to-done times of a finished request. */
int cublox_server_request_times(cublox_server *s, int64_t request_id, double *queued_ms,
                                double *latency_ms);
/* A finished fetch's samples, as cublox_grid_fetch_batch returns them; with
 * out_pos and out_state NULL only n_samples is set.                         */
int cublox_server_fetch_result(cublox_server *s, int64_t request_id, int64_t *offsets,
                               float *out_pos, uint8_t *out_state, int64_t capacity,
                               int64_t *n_samples);
int cublox_server_release(cublox_server *s, int64_t request_id); /* forget */
/* After draining: the map's stored log-odds (dense, reference layout) and
 * window origin.                                                            */
int cublox_server_export(cublox_server *s, int map_id, float *occ_host, int origin_index[3]);
int cublox_server_get_stats(cublox_server *s, cublox_server_stats *out);
/* Withdraw a request still waiting in its map's queue: it ends FAILED with
 * CUBLOX_ERR_CANCELLED and has no effect on the map.  A request the worker
 * has already taken cannot be withdrawn (CUBLOX_ERR_INVALID).  The
 * reference's driver has no queue to withdraw from (main.cpp:464-491).     */
int cublox_server_cancel(cublox_server *s, int64_t request_id);
/* Device bytes a server with this configuration holds besides its maps
 * (tick point buffers, descriptors, fetch scratch): the least usable
 * hbm_budget_bytes.                                                        */
int cublox_server_scratch_bytes(const cublox_server_config *cfg, uint64_t *bytes);

/* ---- allocation-free integration ------------------------------------------
 * No counterpart in the reference: it exists for callers that must not
 * allocate device memory while running (a real-time mapping loop that
 * reserves all GPU memory at start-up, code inside a host framework that is
 * handed only a stream and buffers it owns).  The caller owns every buffer:
 * the map view's occ / cnt / hit arrays (voxel_num elements each, in the
 * ring-buffer hash order; cnt and hit must be zero before the first call
 * and are left zero by every call) and the points, a device array of n x,
 * then n y, then n z.  The call integrates one scan exactly as
 * cublox_grid_update does for the same window origin (there is no
 * first-run origin snap: origin_index is used as given), enqueues on
 * `stream` (a cudaStream_t, NULL for the default stream) and returns.
 *
 * Its only scratch is a fixed area of about 4 MiB in a file-scope device
 * array that every GPU loading this library holds until exit; it allocates
 * nothing and calls no allocating routine.  At most
 * CUBLOX_NOALLOC_MAX_POINTS points per call; more are rejected with
 * CUBLOX_ERR_INVALID.  The first call on each device looks the scratch
 * array's address up (cudaGetSymbolAddress); make that first call before
 * any stream capture.  All calls share the scratch: calls whose GPU work
 * overlaps in time race and give wrong maps.  Errors: the message is in
 * cublox_noalloc_last_error().  There is no device-side error word: the
 * kernels of this path form only in-range indices and have no check that
 * can fail on the device; CUDA launch errors are returned as
 * CUBLOX_ERR_CUDA.                                                         */
#define CUBLOX_NOALLOC_MAX_POINTS 262144

typedef struct {
  float *occ;                /* stored log-odds, device                    */
  uint32_t *cnt;             /* per-scan traversal counters, device        */
  uint32_t *hit;             /* per-scan hit counters, device              */
  int half_map_size[3];
  int origin_index[3];       /* sliding-window origin, global voxel index  */
  float resolution;
  int origin_at_center;
  float max_range;
  float l_hit, l_miss, l_min, l_max;  /* log-odds parameters               */
} cublox_map_view;

int cublox_integrate_noalloc(const cublox_map_view *map, const float *xyz_soa, int n,
                             const float sensor_origin[3], void *stream);
const char *cublox_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* CUBLOX_B200_H */
