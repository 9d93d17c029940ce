// Internal view of a cublox_grid, shared by capi.cu and batch.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "exact_fp.cuh"
#include "kernels.cuh"

namespace cublox_b200 {
// Device scratch of a sphere fetch: the query block (centres | boxes |
// radii | work units | per-unit counts, offsets and limits) and the sample
// outputs.  A grid grows its own on demand; the server owns one, sized when
// it is created, shared by its fetches (they run one at a time).
struct FetchScratch {
  void *fq = nullptr;
  size_t fq_bytes = 0;
  float *fpos = nullptr;
  uint8_t *fstate = nullptr;
  int64_t fcap = 0;
};
}  // namespace cublox_b200

struct cublox_grid {
  // Grid::Config (Grid.hpp:44-53)
  int half[3] = {0, 0, 0};
  int map[3] = {0, 0, 0};
  int voxel_num = 0;
  float res = 0.0f, res_inv = 0.0f;
  bool ctr = false;
  bool has_thr = false;
  float thr_sq = 0.0f;
  int origin_i[3] = {0, 0, 0};
  float origin_f[3] = {0.0f, 0.0f, 0.0f};
  bool first_run = true;
  float max_range = 25.0f;
  // OccupancyGrid.hpp:162-168 defaults
  float l_hit = 0.847f, l_miss = -0.405f, l_min = -1.992f, l_max = 3.476f;
  float l_free = -0.0004f, l_occ = 1.7346f, l_unknown = 0.0f;
  unsigned fp = cublox_b200::kFpPinned;
  int recenter_mode = 0;
  bool stats_on = false;
  // kernel options (cublox_grid_set_option)
  int opt_raycast = 2;  // 0 thread per ray, 1 binned warp walk, 2 split walk
  int opt_seg = 64;     // split walk: target in-window steps per lane
  int opt_fold = 2;     // 0 scalar sweep, 1 vector sweep, flagged lines: 2 lists, 3 per warp
  int opt_block = 512;  // split walk CTA size
  int opt_contig = 0;   // split walk: contiguous segment runs per CTA
  int opt_cube = 32;    // shared-memory counter cube side (0, 16, 32)
  bool opt_flat = false;  // split walk, cube 32: 32 x 32 x 16 (CUBLOX_OPT_FLAT_CUBE)
  int opt_match = 0;    // merge duplicate voxels within a warp
  int opt_sort = 0;     // walk rays in direction-bin order
  void *d_segs = nullptr;  // split walk: segment records
  void *d_rays = nullptr;  // split walk: ray records
  int *d_work = nullptr;   // split walk: 2 counters
  int split_cap = 0;       // rays the split scratch holds
  int *d_bins = nullptr;
  int *d_hist = nullptr;
  float *d_sorted = nullptr;
  int bin_cap = 0;
  bool timing_on = false;
  int64_t last_cleared = 0;  // voxels the last recenter cleared
  cudaEvent_t tev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool tev_used[3] = {false, false, false};

  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  // voxel layout of occ / cnt / hit (brick sides, strides) and the voxels
  // each array holds: the largest padded size of the layouts a grid can
  // switch between, a multiple of 32, so a layout change needs no new memory
  cublox_b200::VoxLayout lay{};
  int lay_code = 0;     // brick sides as log2 digits x y z (320: 8 x 4 x 1)
  int64_t nalloc = 0;
  int nlines = 0;       // nalloc / 32
  uint8_t *d_dirty = nullptr;  // line flags (kernels.cuh)
  int nbr[3] = {0, 0, 0};      // bricks per axis in the current layout

  float *d_occ = nullptr;
  uint32_t *d_cnt = nullptr;
  uint32_t *d_hit = nullptr;
  unsigned long long *d_stats = nullptr;  // 4
  uint32_t *d_err = nullptr;
  uint32_t *d_masks = nullptr;  // recenter slab masks
  uint32_t *h_masks = nullptr;  // pinned staging of the masks, two halves
  cudaEvent_t mask_ev[2] = {nullptr, nullptr};  // a half free again
  int mask_half = 0;  // the half the next recenter stages into
  int mask_stage_words = 0;  // words per half: slab masks + brick lists
  int mask_words[3] = {0, 0, 0};

  float *d_cloud = nullptr;  // SoA [x|y|z]
  int cloud_cap = 0;
  float *d_world = nullptr;  // update_pose: world-frame SoA points
  int world_cap = 0;
  int *d_kept = nullptr;     // update_pose: points kept by the range filter
  unsigned char *d_image = nullptr;  // update_depth: the image on the device
  size_t image_cap = 0;
  float *h_stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int stage_cap = 0;
  int stage_idx = 0;

  cublox_b200::FetchScratch fs;  // fetch scratch, grown on demand
  uint8_t *d_qout = nullptr;
  float *d_qin = nullptr;
  int qcap = 0;
};

namespace cublox_b200 {
namespace detail {
// Every device and pinned-host allocation and free this library makes goes
// through these, which count them (cublox_runtime_counters), so that a
// caller can check that a steady state allocates nothing.
enum Counter { kDevAllocs = 0, kDevFrees, kPinnedAllocs, kPinnedFrees, kGraphBuilds, kNumCounters };
void count(Counter c);
cudaError_t dev_alloc(void **p, size_t bytes);
cudaError_t dev_free(void *p);
cudaError_t pinned_alloc(void **p, size_t bytes);
cudaError_t pinned_free(void *p);
template <class T>
inline cudaError_t dmalloc(T **p, size_t bytes) {
  return dev_alloc(reinterpret_cast<void **>(p), bytes);
}
template <class T>
inline cudaError_t hmalloc(T **p, size_t bytes) {
  return pinned_alloc(reinterpret_cast<void **>(p), bytes);
}
inline cudaError_t dfree(const void *p) { return dev_free(const_cast<void *>(p)); }
inline cudaError_t hfree(const void *p) { return pinned_free(const_cast<void *>(p)); }

int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what, int line);
// The default voxel layout of new grids (log2 brick sides as digits x y z)
// and the layouts a grid may switch to: 32-voxel bricks and the reference's
// hash order (0).
constexpr int kDefaultLayout = 320;
constexpr int kLayouts[] = {320, 230, 221, 0};
bool layout_valid(int code);
// Device bytes of a grid's voxel arrays and line flags (its largest layout).
size_t voxel_bytes_for(const int half[3]);
// Switch a grid's arrays to another layout, moving its stored log-odds
// (counters are zero between scans).  Enqueued on the grid's stream.
int set_layout(cublox_grid *g, int code);
// Stored log-odds in the reference's hash order from a copy of the grid's
// occ array in its own layout (host memory, nalloc values).
void layout_to_reference(const cublox_grid *g, const float *arr, float *ref);
// First update: snap the window origin to the sensor voxel
// (OccupancyGrid.cpp:192-198).
void snap_first_run(cublox_grid *g, const float sensor[3]);
// RayParams of one scan on this grid (points and counters filled in).
RayParams ray_params(const cublox_grid *g, const float *x, const float *y, const float *z,
                     int n, int stride, const float sensor[3]);
// Device memory a grid holds now: voxel buffers plus the per-call scratch
// it has grown.
size_t device_bytes(const cublox_grid *g);
// Free the per-call scratch a grid has grown (cloud staging, walk plans,
// fetch and query buffers); the voxel buffers stay.  Syncs the grid's
// stream.
int release_scratch(cublox_grid *g);
// Allocate the voxel buffers of a grid whose buffers were detached
// (detach_voxels), stored log-odds from occ_host (all unknown if null),
// counters zero.
int acquire_device(cublox_grid *g, const float *occ_host);
// A grid's voxel buffers (stored log-odds, traversal and hit counters)
// detached from it, to be handed to another grid of the same allocation
// size without freeing and allocating.  The counters are zero (they are
// between scans).
struct VoxelBuffers {
  int64_t nalloc = 0;
  float *occ = nullptr;
  uint32_t *cnt = nullptr, *hit = nullptr;
  size_t bytes() const { return 12 * static_cast<size_t>(nalloc); }
};
// Voxels the arrays of a grid with these half sizes hold (padding included).
int64_t nalloc_for(const int half[3]);
// Detach g's voxel buffers into *out after enqueueing, on g's stream, the
// copy of its stored log-odds to occ_host (pinned for the copy to be
// asynchronous).  No sync, no free.  g must not be used until attach_voxels.
int detach_voxels(cublox_grid *g, float *occ_host, VoxelBuffers *out);
// Give g the buffers *in (same nalloc) and enqueue, on g's stream, the copy
// of its stored log-odds from occ_host (all unknown if null).
int attach_voxels(cublox_grid *g, VoxelBuffers *in, const float *occ_host);
// fetch_batch on stream st (ordered after the grid's work by the caller),
// outputs sized to the samples found, in the scratch `sc` (the grid's own if
// null).
int fetch_into(cublox_grid *g, cudaStream_t st, const float *centers, int nq, float radius,
               int filter, int max_results, std::vector<int64_t> &offsets,
               std::vector<float> &pos, std::vector<uint8_t> &state,
               FetchScratch *sc = nullptr);
// Size `sc` for fetches of up to `centres` centres and `samples` samples, so
// that such fetches allocate nothing.
int reserve_fetch(FetchScratch *sc, int centres, int64_t samples, cudaStream_t st);
void free_fetch(FetchScratch *sc);
}  // namespace detail
}  // namespace cublox_b200
