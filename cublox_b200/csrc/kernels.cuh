// Device kernels of the map-integration path.
//
// Grid storage (one map), every array in the same voxel layout (VoxLayout):
//   occ    float[A]   stored log-odds
//   cnt    uint32[A]  per-scan traversal count (bits 0..30) and a "has hit"
//                     flag (bit 31); zero between scans
//   hit    uint32[A]  per-scan endpoint-hit count, read only where flagged
//   dirty  uint8[A/32]  per 32-voxel line of the arrays: 1 if the scan being
//                     integrated has counted a voxel of the line; zero
//                     between scans
// A voxel's ring-buffer slot per axis is s = l + h (local index l in
// [-h, h], utils.cuh:60-70), as in the reference's hash
// ((sx*ny + sy)*nz + sz) (utils.cuh:131-136).
#pragma once

#include <cstdint>

#include "exact_fp.cuh"

namespace cublox_b200 {

constexpr uint32_t kHitFlag = 0x80000000u;
constexpr uint32_t kOpMask = 0x7fffffffu;
constexpr int kLineShift = 5;  // 32 voxels (128 bytes of one array) per line

// Where a voxel lives in a map's arrays.  The slots are cut into bricks of
// 2^lb[0] x 2^lb[1] x 2^lb[2] voxels stored one after another (brick index
// x-major, z fastest), voxels inside a brick x-major too, so the address is
// a sum of one term per axis:
//   addr = sum_a (s_a >> lb[a]) * bs[a] + (s_a & (2^lb[a] - 1)) * is[a].
// lb = {0, 0, 0} is the reference's hash order.  With 32-voxel bricks
// (lb summing to 5) a brick is one 128-byte line: a ray crossing a brick
// touches one line, and the fold reads and writes whole lines.
struct VoxLayout {
  int lb[3];  // log2 brick side per axis
  int bs[3];  // address step of one brick along the axis
  int is[3];  // address step of one voxel inside a brick along the axis
};

CBX_HD int vox_axis(const VoxLayout &L, int a, int s) {
  return (s >> L.lb[a]) * L.bs[a] + (s & ((1 << L.lb[a]) - 1)) * L.is[a];
}

CBX_HD int vox_addr(const VoxLayout &L, int sx, int sy, int sz) {
  return vox_axis(L, 0, sx) + vox_axis(L, 1, sy) + vox_axis(L, 2, sz);
}

// Error-word bits (never expected; set instead of trapping).
constexpr uint32_t kErrHashRange = 1u << 0;
constexpr uint32_t kErrFetchOverflow = 1u << 1;
constexpr uint32_t kErrJumpStall = 1u << 2;
constexpr uint32_t kErrWaitTimeout = 1u << 3;  // fused batch launch: a fold wait gave up

struct RayParams {
  const float *x, *y, *z;  // point i is (x[i*stride], y[i*stride], z[i*stride])
  int n;
  int stride;
  float o[3];       // sensor origin (world)
  int win[3];       // sliding-window origin (global voxel index)
  int half[3], map[3];
  float res, inv, max_range;
  int vnum;
  int ctr;
  unsigned fp;
  uint32_t *cnt;
  uint32_t *hit;
  unsigned long long *stats;  // [rays, op_incs, hit_incs] or null
  uint32_t *err;
  VoxLayout lay;
  uint8_t *dirty;  // line flags to set, or null (the fold sweeps every line)
};

struct ApplyParams {
  float *occ;
  uint32_t *cnt;
  uint32_t *hit;
  int vnum;    // voxels swept by the full sweep (variants 0, 1)
  float l_hit, l_miss, l_min, l_max, l_unknown;
  unsigned fp;
  unsigned long long *stats;  // [3] += touched
  int variant;                // 0 scalar sweep, 1 vector sweep, 2 flagged lines
                              // (per-CTA line lists), 3 flagged lines (per warp)
  uint8_t *dirty;             // variants 2, 3: line flags (cleared as folded)
  int nlines;                 // variants 2, 3: lines
  uint32_t *err;              // error word (a bounded wait that gave up)
};

struct ClearParams {
  float *occ;
  const uint32_t *xmask, *ymask, *zmask;  // bit per local slab slot
  int map[3];
  int any_z;
  int x_done;  // marked x slabs are already cleared (contiguous memsets)
  VoxLayout lay;
  // brick layouts: the bricks to visit, as three lists (brick index along x,
  // y, z of a brick column, row or level that holds a marked slab), each
  // crossed with every brick of the other two axes
  const int *blist;  // nb[0] x indices, nb[1] y indices, nb[2] z indices
  int nb[3];
  int nbr[3];        // bricks per axis
};

// A fetch's candidates are cut into work units of `unit` consecutive
// candidates of one query (in the query's (x, y, z) order), so that one
// large sphere spreads over the whole GPU while many small ones stay whole.
constexpr int kFetchMinUnit = 8192;

struct FetchParams {
  const float *occ;
  const float *centers;  // 3 per query
  const int *qbox;       // 8 ints per query: gx0 gx1 gy0 gy1 gz0 gz1 pad pad
  const float *qr2;      // radius_sq per query
  int nq;
  const int *uq;             // per unit: its query
  const long long *ut0;      // per unit: its first candidate
  int nu;
  long long unit;            // candidates per unit
  int win[3], half[3], map[3];
  float res;
  int ctr;
  unsigned fp;
  float l_free, l_occ, l_unknown;
  int filter;
  VoxLayout lay;
  long long *counts;         // pass 1 output: samples per unit
  const long long *offsets;  // pass 2 input: where each unit's samples go
  const long long *limits;   // pass 2: samples each unit keeps (the cap)
  float *out_pos;
  uint8_t *out_state;
  uint32_t *err;
};

struct QueryParams {
  const float *occ;
  const float *xyz;
  int n;
  int win[3], half[3], map[3];
  float inv;
  int ctr;
  float l_free, l_occ, l_unknown;
  uint8_t *out;
  VoxLayout lay;
};

// Copy between a map's layout and the reference's hash order (export,
// import): to_ref = 1 writes ref[h] = arr[addr(h)], else arr[addr(h)] =
// ref[h], for every voxel h of the map.
void launch_relayout(const float *src, float *dst, const VoxLayout &lay, const int map[3],
                     int to_ref, cudaStream_t s);

void launch_raycast(const RayParams &p, cudaStream_t s);

// Scratch of the direction-binned raycast (raycast_binned.cu).
struct BinnedScratch {
  int *bins;      // per ray
  int *hist;      // binned_bins()
  int *cursor;    // binned_bins()
  float *sorted;  // 3 * n (SoA)
};
int binned_bins();
// Counting sort of the rays by octahedral direction bin into b.sorted (SoA).
void launch_direction_sort(const RayParams &p, const BinnedScratch &b, cudaStream_t s);
// Warp-cooperative exact walk (raycast_split.cu): rays longer than seg_len
// in-window steps are cut into time segments walked by separate lanes.
struct SplitScratch {
  void *segs;     // seg_cap segment records (split_seg_bytes() each)
  void *rays;     // n ray records (split_ray_bytes() each)
  int *counters;  // 2 ints: segments planned, work queue
  int seg_cap;
  int max_segs;   // per ray
  int block;      // walk CTA size (256, 512 or 1024)
  int contiguous; // 1: each CTA walks one contiguous run of segments
};
size_t split_seg_bytes();
size_t split_ray_bytes();
// cube: side of the shared-memory counter cube (0, 8, 16, 32); flat (cube
// 32 only): a 32 x 32 x 16 cube, two CTAs per SM.
void launch_raycast_split(const RayParams &p, int cube, bool flat, int seg_len,
                          const SplitScratch &sc, cudaStream_t s);
// cube: side of the shared-memory counter cube (16 or 32); match: merge
// duplicate voxel keys within a warp; sort: walk rays in direction order.
void launch_raycast_binned(const RayParams &p, const BinnedScratch &b, int cube,
                           bool match, bool sort, cudaStream_t s);
// The loaded kernels' binary version on the current device (100 for
// sm_100a), -1 if it cannot be read.
int kernel_binary_version();
// Accounting: stats[0] += the reference loop's iterations + 1 per ray.
void launch_step_count(const RayParams &p, cudaStream_t s);
void launch_apply(const ApplyParams &p, cudaStream_t s);
void launch_clear(const ClearParams &p, cudaStream_t s);
void launch_fetch(const FetchParams &p, int pass, cudaStream_t s);
void launch_query(const QueryParams &p, cudaStream_t s);
// Sensor-frame cloud -> world-frame SoA (the reference driver's
// buildCloudInOdomFrame, src/main.cpp:640-693): non-finite points and points
// farther than sqrt(max_r2) from the sensor are dropped (written as NaN, which
// the walk drops), the rest become R p + t.
struct IngestParams {
  const float *xyz;  // points, layout 0 SoA (columns `col` floats apart) / 1 AoS
  int layout, n;     // the first n points are used
  int col;
  float R[9];        // row-major rotation, sensor -> world
  float t[3];        // sensor origin in the world
  float max_r2;      // squared range filter
  float *dst;        // SoA world points
  int *count;        // if not null: += points kept
};
void launch_ingest(const IngestParams &p, cudaStream_t s);

// Depth image -> sensor-frame points (the reference driver's depthCallback,
// src/main.cpp:558-632), then the same filter and transform as IngestParams,
// one pixel per point (row-major), written as world-frame SoA.
struct DepthParams {
  const unsigned char *image;  // height rows of `step` bytes
  int encoding;                // 0: 16-bit millimetres (16UC1, mono16), 1: 32-bit float metres
  int width, height;
  long long step;
  float fx, fy, cx, cy;
  IngestParams ingest;         // xyz, layout unused; n = width * height
};
void launch_depth(const DepthParams &p, cudaStream_t s);

// Visualisation cloud of fetch samples (the reference driver's
// publishOccupancyCloudAsync, src/main.cpp:740-790): samples in order,
// dropped by the global-index subsample hash, coloured by distance to the
// robot, packed as x, y, z, rgb floats, at most max_points written.
struct VizParams {
  const float *pos;  // n samples, x0 y0 z0 x1 ...
  long long n;
  float inv;
  int ctr;
  int step;          // subsample: keep 1 of `step` (<= 1: all)
  float d_max;       // colour scale (max_viz_radius)
  float o[3];        // robot position
  long long max_points;
  float *out;        // 4 floats per written point
  long long *written;
};
void launch_viz(const VizParams &p, cudaStream_t s);

void launch_gather_soa(const float *xyz, int layout, int n, float *dst,
                       cudaStream_t s);

}  // namespace cublox_b200
