/*
 * cublox CPU oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, scalar restatement of the reference's map-integration path
 * (mrsp/cublox), used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  Nothing in the product (cublox_b200/,
 * include/) links, imports or calls this code.
 *
 * Every FP32 operation is spelled out in the reference's order.  The file is
 * compiled with -ffp-contract=off, so no multiply-add is fused unless the
 * code calls fmaf() explicitly.  Which multiply-adds the reference's device
 * build fuses is selected by the ORC_FP_* bits of `fp_mode`; the pinned
 * combination is ORC_FP_PINNED (decided black-box against the reference's
 * own sm_100a build, see tests/test_contraction_pins.py).
 *
 * Host-side arithmetic of the reference (Eigen on x86-64 g++, no FMA) is
 * restated with plain float ops.
 */
#ifndef CUBLOX_ORACLE_H
#define CUBLOX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- contraction-site selectors (bit fields of fp_mode) ---------------- */
/* sum-of-squares shapes for  x*x + y*y + z*z                               */
#define ORC_SOS_PLAIN 0 /* (x*x + y*y) + z*z                               */
#define ORC_SOS_FY_FZ 1 /* fma(z,z, fma(y,y, x*x))                          */
#define ORC_SOS_FX_FZ 2 /* fma(z,z, fma(x,x, y*y))                          */
#define ORC_SOS_P_FZ 3  /* fma(z,z, x*x + y*y)                              */
#define ORC_SOS_FY_P 4  /* fma(y,y, x*x) + z*z                              */
#define ORC_SOS_FX_P 5  /* fma(x,x, y*y) + z*z                              */

#define ORC_FP_RAY_SOS_SHIFT 0   /* 3 bits: ray length  kernels.cu:50       */
#define ORC_FP_CLIP_FMA (1u << 3)   /* e = o + d*s        kernels.cu:60-62  */
#define ORC_FP_BOUND_FMA (1u << 4)  /* b*res - o          kernels.cu:89-100 */
#define ORC_FP_CENTER_FMA (1u << 5) /* p*inv + s*0.5      utils.cuh:27-29   */
#define ORC_FP_MISS_FMA (1u << 6)   /* l += l_miss*miss   kernels.cu:188    */
#define ORC_FP_HIT_FMA (1u << 7)    /* l += l_hit*hit     kernels.cu:189    */
#define ORC_FP_REC_SOS_SHIFT 8      /* 3 bits: recenter gate kernels.cu:329 */
#define ORC_FP_FETCH_SOS_SHIFT 11   /* 3 bits: fetch sphere kernels.cu:535  */
#define ORC_FP_FETCH_DFMA (1u << 14) /* pos - c, pos = t*res kernels.cu:532 */

#define ORC_FP_RAY_SOS(m) (((m) >> ORC_FP_RAY_SOS_SHIFT) & 7u)
#define ORC_FP_REC_SOS(m) (((m) >> ORC_FP_REC_SOS_SHIFT) & 7u)
#define ORC_FP_FETCH_SOS(m) (((m) >> ORC_FP_FETCH_SOS_SHIFT) & 7u)

/* Pinned device contraction pattern of the reference's sm_100a build.      */
/* Pinned on the reference built for sm_100a with its release flags:      */
/* sums of squares fma(z,z, fma(x,x, y*y)); apply terms fused; clip point, */
/* boundary distance and fetch offset not fused.  Centre binning: fused    */
/* and unfused agree except at exact ties of p*inv (no input separates     */
/* them), so the fused reading is kept.                                    */
#define ORC_FP_PINNED                                                        \
  ((ORC_SOS_FX_FZ << ORC_FP_RAY_SOS_SHIFT) | ORC_FP_CENTER_FMA |            \
   ORC_FP_MISS_FMA | ORC_FP_HIT_FMA | (ORC_SOS_FX_FZ << ORC_FP_REC_SOS_SHIFT) | \
   (ORC_SOS_FX_FZ << ORC_FP_FETCH_SOS_SHIFT))

/* ---- grid state (mirrors Grid + OccupancyGrid members) ------------------ */
typedef struct {
  int half[3];
  int map[3];
  int voxel_num;
  float res, res_inv;
  int origin_at_center;
  int has_thr;
  float thr, thr_sq;
  int origin_i[3];
  float origin_f[3];
  int first_run;
  float max_range;
  float l_hit, l_miss, l_min, l_max, l_free, l_occ, l_unknown;
  unsigned fp_mode;
  float *occ;
  int *op;
  int *hit;
} orc_grid;

typedef struct {
  int64_t rays;        /* points that were not dropped                    */
  int64_t voxel_steps; /* DDA iterations that did not break + 1 endpoint  */
  int64_t op_incs;     /* in-window op increments (U)                      */
  int64_t hit_incs;    /* hit increments (H)                               */
  int64_t touched;     /* voxels with op > 0 at apply time (T)             */
} orc_stats;

/* Returns 0 on success, -1 if the voxel count exceeds int32 (Grid.cpp:44). */
int orc_grid_init(orc_grid *g, const int half[3], float res,
                  int origin_at_center, int has_thr, double thr,
                  const float origin[3]);
void orc_grid_free(orc_grid *g);
void orc_grid_reset(orc_grid *g);
void orc_set_log_odds(orc_grid *g, float l_hit, float l_miss, float l_min,
                      float l_max, float l_free, float l_occ);
void orc_set_max_range(orc_grid *g, float r);
void orc_set_fp_mode(orc_grid *g, unsigned mode);
void orc_set_origin_i(orc_grid *g, const int origin_i[3]);

/* Index math (utils.cuh / utils.hpp).  host=1 selects the host compiler's
 * rounding (no FMA, x86 truncation); host=0 the device's.                  */
int orc_pos_to_global(float p, float res_inv, int origin_at_center, int host,
                      unsigned fp_mode);
int orc_global_to_local(int g, int map, int half);
int orc_local_to_global(int l, int map, int half, int origin);
int orc_global_to_hash(const int g[3], const int map[3], const int half[3]);
void orc_hash_to_local(int h, const int map[3], const int half[3], int l[3]);
float orc_global_to_pos(int g, float res, int origin_at_center);
float orc_logit(float p);

/* The reference driver's buildCloudInOdomFrame (src/main.cpp:640-693): keep
 * finite points with (x*x + y*y) + z*z <= max_r2, write ((r0*x + r1*y) +
 * r2*z) + t per row (Eigen's order for Isometry3f * Vector3f on x86-64
 * without FMA; R row-major), in input order.  Returns the points kept.
 * Eigen itself is absent here, so that order is restated, not pinned.     */
int orc_ingest(const float *xyz_aos, int n, const float R[9], const float t[3],
               float max_r2, float *out_aos);

/* The reference driver's depthCallback (src/main.cpp:558-632): one
 * camera-frame point per pixel (row-major) of a 16-bit millimetre
 * (encoding 0) or float metre (1) image, NaN where the depth is invalid.
 * K = {fx, fy, cx, cy}.                                                   */
void orc_depth_cloud(const unsigned char *image, int encoding, int width, int height,
                     long long step, const float K[4], float *out_aos);

/* The driver's visualisation cloud of fetch samples (src/main.cpp:740-790):
 * x, y, z, rgb per kept sample, in sample order.  Returns the count.      */
long long orc_viz(const float *pos, long long n, float inv, int ctr, int step, float d_max,
                  long long max_points, const float robot[3], float *out);

/* Raycast of one scan into op/hit (kernels.cu:33-152).  Does not snap the
 * first-run origin and does not apply.  `nthreads` > 1 splits the rays over
 * POSIX threads with relaxed atomic increments.                            */
void orc_raycast(orc_grid *g, const float *x, const float *y, const float *z,
                 int n, const float sensor[3], orc_stats *st, int nthreads);
/* Voxel steps of one scan (the reference loop's iterations that did not
 * break + 1 endpoint per kept ray), with no grid: the count does not depend
 * on the window.  res_inv is 1 / res as Grid.cpp computes it.              */
int64_t orc_count_steps(float res, int origin_at_center, float max_range, unsigned fp_mode,
                        const float *x, const float *y, const float *z, int n,
                        const float sensor[3], int nthreads);
/* Fold counters into occ and zero them (kernels.cu:167-210).               */
void orc_apply(orc_grid *g, orc_stats *st, int nthreads);
/* OccupancyGrid::update (OccupancyGrid.cpp:181-238).                       */
void orc_update(orc_grid *g, const float *x, const float *y, const float *z,
                int n, const float sensor[3], orc_stats *st, int nthreads);

/* Trace one ray: the in-window hashes it increments, in order, the endpoint
 * last (flagged through *end_hit = 1 if it also counts a hit).  Returns the
 * number written (<= cap), or -1 if the ray is dropped.                    */
int orc_trace_ray(const orc_grid *g, float ex, float ey, float ez,
                  const float sensor[3], int *out, int cap, int *n_total,
                  int *end_in_window, int *end_hit);

/* OccupancyGrid::recenter (OccupancyGrid.cpp:141-179 + kernels.cu:313-499).
 * compat=1 clears the reference's extra "entering" band.  Returns the
 * action (0 none, 1 slabs, 2 full reset).  slabs[a] (capacity map[a]) gets
 * the distinct local slab indices cleared on axis a, ascending.            */
int orc_recenter(orc_grid *g, const float pos[3], int compat, int *host_skip,
                 int new_origin[3], int *slabs[3], int n_slabs[3]);

/* OccupancyGrid::fetchOccupancyAround (OccupancyGrid.cpp:240-356 +
 * kernels.cu:506-562).  Samples are produced in (gx, gy, gz) ascending
 * order; the first min(count, cap) are written.  Returns the number
 * written; *n_pass = voxels passing the sphere+filter tests.              */
int64_t orc_fetch(const orc_grid *g, const float center[3], float radius,
                  int filter, int max_results, float *out_pos,
                  uint8_t *out_state, int64_t out_cap, int64_t *n_pass);

/* Probe search: indices of rays whose trace differs between two patterns. */
int orc_find_trace_diff(const orc_grid *g, unsigned mode_a, unsigned mode_b,
                        const float *pts, int n, const float sensor[3],
                        int *out_idx, int cap);

/* x*x + y*y + z*z in one of the ORC_SOS_* shapes.                          */
float orc_sos(float x, float y, float z, unsigned shape);

/* The fetch kernel's sphere-test sum for voxel gi about centre c.          */
float orc_fetch_sos(const float c[3], const int gi[3], float res, int ctr,
                    unsigned mode);

/* Point queries (OccupancyGrid.cpp:358-429).  Returns 0/1.                 */
int orc_is_state_pos(const orc_grid *g, const float pos[3], int state);

#ifdef __cplusplus
}
#endif
#endif
