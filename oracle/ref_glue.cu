/*
 * Reference harness — TEST / BASELINE INFRASTRUCTURE ONLY.
 *
 * Host glue that drives the reference's own device code (its src/kernels.cu,
 * compiled from the reference tree by oracle/Makefile into oracle/_ref/) in
 * the same sequence as the reference's OccupancyGrid host class
 * (src/OccupancyGrid.cpp), which cannot be built here because it needs
 * Eigen.  The sequence replicated per call:
 *   ctor      OccupancyGrid.cpp:54-65   + Grid.cpp:27-54, allocate :431-480
 *   update    OccupancyGrid.cpp:181-238 (3 pageable H2D copies on stream 0,
 *             raycast, sync, full-grid apply, sync)
 *   recenter  OccupancyGrid.cpp:141-179 (host gate, launchRecenter)
 *   fetch     OccupancyGrid.cpp:240-356 (host bounds, one launch, device
 *             sync, D2H count + samples)
 * Host arithmetic is plain float (x86-64, no FMA), as the reference's g++
 * build computes it.
 */
#include <cublox/kernels.hpp>

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>

namespace {

int host_p2g(float p, float inv, bool ctr) {
  if (ctr) {
    const float s = p < 0.0f ? -1.0f : 1.0f;
    return static_cast<int>(p * inv + s * 0.5f);
  }
  return static_cast<int>(std::floor(p * inv));
}

float host_g2p(int g, float res, bool ctr) {
  return ctr ? g * res : (g + 0.5f) * res;
}

struct RefGrid {
  int half[3];
  int map[3];
  int voxel_num;
  float res, res_inv;
  bool ctr;
  bool has_thr;
  float thr_sq;
  int origin_i[3];
  float origin_f[3];
  bool first_run;
  float max_range;
  float l_hit, l_miss, l_min, l_max, l_free, l_occ, l_unknown;
  int *d_op, *d_hit;
  float *d_occ;
  int *d_slices[3];
  cublox::RecenterResult *d_result;
  float *d_x, *d_y, *d_z;
  int cloud_cap;
  unsigned *d_fcount;
  float3 *d_fpos;
  unsigned char *d_fstate;
  int fetch_cap;
};

void set_origin(RefGrid *g, const int o[3]) {
  for (int a = 0; a < 3; ++a) {
    g->origin_i[a] = o[a];
    g->origin_f[a] = host_g2p(o[a], g->res, g->ctr);
  }
}

#define CK(call)                                                             \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      std::fprintf(stderr, "ref_glue: %s -> %s (%s:%d)\n", #call,            \
                   cudaGetErrorString(e_), __FILE__, __LINE__);              \
      return -1;                                                             \
    }                                                                        \
  } while (0)

} // namespace

extern "C" {

int ref_pageable_access(int dev) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrPageableMemoryAccess, dev) !=
      cudaSuccess)
    return -1;
  return v;
}

void ref_destroy(void *hp) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  if (!g) return;
  cudaFree(g->d_op);
  cudaFree(g->d_hit);
  cudaFree(g->d_occ);
  for (int a = 0; a < 3; ++a) cudaFree(g->d_slices[a]);
  cudaFree(g->d_result);
  cudaFree(g->d_x);
  cudaFree(g->d_y);
  cudaFree(g->d_z);
  cudaFree(g->d_fcount);
  cudaFree(g->d_fpos);
  cudaFree(g->d_fstate);
  delete g;
}

int ref_create(const int half[3], float res, int origin_at_center,
               int has_thr, double thr, const float origin[3], void **out) {
  RefGrid *g = new RefGrid();
  std::memset(g, 0, sizeof(RefGrid));
  g->res = res;
  g->res_inv = 1.0f / res;
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    g->half[a] = half[a];
    g->map[a] = 2 * half[a] + 1;
    total *= g->map[a];
  }
  if (total > std::numeric_limits<int>::max()) {
    delete g;
    return -2;
  }
  g->voxel_num = static_cast<int>(total);
  g->has_thr = has_thr != 0;
  if (g->has_thr) {
    const float t = static_cast<float>(thr);
    g->thr_sq = t * t;
  }
  g->ctr = origin_at_center != 0;
  int o[3];
  for (int a = 0; a < 3; ++a) o[a] = host_p2g(origin[a], g->res_inv, g->ctr);
  set_origin(g, o);
  g->first_run = true;
  g->max_range = 25.0f;
  g->l_hit = 0.847f;
  g->l_miss = -0.405f;
  g->l_min = -1.992f;
  g->l_max = 3.476f;
  g->l_free = -0.0004f;
  g->l_occ = 1.7346f;
  g->l_unknown = 0.0f;
  const size_t n = static_cast<size_t>(g->voxel_num);
  if (cudaMalloc(&g->d_op, n * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&g->d_hit, n * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&g->d_occ, n * sizeof(float)) != cudaSuccess ||
      cudaMemset(g->d_op, 0, n * sizeof(int)) != cudaSuccess ||
      cudaMemset(g->d_hit, 0, n * sizeof(int)) != cudaSuccess ||
      cudaMemset(g->d_occ, 0, n * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&g->d_result, sizeof(cublox::RecenterResult)) !=
          cudaSuccess) {
    ref_destroy(g);
    return -1;
  }
  for (int a = 0; a < 3; ++a) {
    if (cudaMalloc(&g->d_slices[a], sizeof(int) * g->map[a]) != cudaSuccess) {
      ref_destroy(g);
      return -1;
    }
  }
  *out = g;
  return 0;
}

void ref_set_max_range(void *hp, float r) {
  static_cast<RefGrid *>(hp)->max_range = r;
}

void ref_set_log_odds(void *hp, float l_hit, float l_miss, float l_min,
                      float l_max, float l_free, float l_occ) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  g->l_hit = l_hit;
  g->l_miss = l_miss;
  g->l_min = l_min;
  g->l_max = l_max;
  g->l_free = l_free;
  g->l_occ = l_occ;
  g->l_unknown = 0.0f;
}

void ref_set_origin_i(void *hp, const int o[3]) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  set_origin(g, o);
  g->first_run = false;
}

void ref_get_origin(void *hp, int o[3], float of[3]) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  for (int a = 0; a < 3; ++a) {
    o[a] = g->origin_i[a];
    of[a] = g->origin_f[a];
  }
}

static int ensure_cloud(RefGrid *g, int n) {
  if (n <= g->cloud_cap) return 0;
  if (g->d_x) {
    CK(cudaFree(g->d_x));
    CK(cudaFree(g->d_y));
    CK(cudaFree(g->d_z));
  }
  g->cloud_cap = n;
  const size_t b = sizeof(float) * static_cast<size_t>(n);
  CK(cudaMalloc(&g->d_x, b));
  CK(cudaMalloc(&g->d_y, b));
  CK(cudaMalloc(&g->d_z, b));
  return 0;
}

/* raycast pass only (counters keep accumulating; no apply). */
int ref_raycast_only(void *hp, const float *x, const float *y, const float *z,
                     int n, const float sensor[3]) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  if (g->voxel_num <= 0 || n <= 0) return 0;
  if (ensure_cloud(g, n)) return -1;
  const size_t b = sizeof(float) * static_cast<size_t>(n);
  CK(cudaMemcpyAsync(g->d_x, x, b, cudaMemcpyHostToDevice, 0));
  CK(cudaMemcpyAsync(g->d_y, y, b, cudaMemcpyHostToDevice, 0));
  CK(cudaMemcpyAsync(g->d_z, z, b, cudaMemcpyHostToDevice, 0));
  cublox::RayCastCfg cfg{};
  cfg.origin = make_float3(sensor[0], sensor[1], sensor[2]);
  cfg.origin_i = make_int3(g->origin_i[0], g->origin_i[1], g->origin_i[2]);
  cfg.map_size_i = make_int3(g->map[0], g->map[1], g->map[2]);
  cfg.half_map_size_i = make_int3(g->half[0], g->half[1], g->half[2]);
  cfg.resolution = g->res;
  cfg.inv_resolution = g->res_inv;
  cfg.max_range = g->max_range;
  cfg.map_vox_num = g->voxel_num;
  cfg.origin_at_center = g->ctr;
  cublox::launchRayCastUpdate(cfg, g->d_x, g->d_y, g->d_z, n, 0, g->d_op,
                              g->d_hit);
  CK(cudaStreamSynchronize(0));
  CK(cudaGetLastError());
  return 0;
}

int ref_apply_only(void *hp) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  cublox::launchApplyUpdate(g->d_occ, g->d_op, g->d_hit, g->voxel_num,
                            g->l_hit, g->l_miss, g->l_min, g->l_max,
                            g->l_unknown, 0);
  CK(cudaStreamSynchronize(0));
  CK(cudaGetLastError());
  return 0;
}

int ref_update(void *hp, const float *x, const float *y, const float *z,
               int n, const float sensor[3]) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  if (g->voxel_num <= 0 || n <= 0) return 0;
  if (g->first_run) {
    int o[3];
    for (int a = 0; a < 3; ++a) o[a] = host_p2g(sensor[a], g->res_inv, g->ctr);
    set_origin(g, o);
    g->first_run = false;
  }
  if (ref_raycast_only(hp, x, y, z, n, sensor)) return -1;
  return ref_apply_only(hp);
}

/* OccupancyGrid::recenter.  *action: 0/1/2; *host_skip = 1 if the host gate
 * returned before any device work. */
int ref_recenter(void *hp, const float pos[3], int *action, int *host_skip,
                 int new_origin[3]) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  *action = 0;
  *host_skip = 1;
  for (int a = 0; a < 3; ++a) new_origin[a] = g->origin_i[a];
  if (!g->has_thr) return 0;
  const float dx = pos[0] - g->origin_f[0];
  const float dy = pos[1] - g->origin_f[1];
  const float dz = pos[2] - g->origin_f[2];
  const float sq = (dx * dx + dy * dy) + dz * dz;
  if (sq < g->thr_sq) return 0;
  *host_skip = 0;
  cublox::RecenterCfg cfg{};
  cfg.pos = make_float3(pos[0], pos[1], pos[2]);
  cfg.origin_f = make_float3(g->origin_f[0], g->origin_f[1], g->origin_f[2]);
  cfg.origin_i = make_int3(g->origin_i[0], g->origin_i[1], g->origin_i[2]);
  cfg.map_size_i = make_int3(g->map[0], g->map[1], g->map[2]);
  cfg.half_map_size_i = make_int3(g->half[0], g->half[1], g->half[2]);
  cfg.resolution = g->res;
  cfg.inv_resolution = g->res_inv;
  cfg.recenter_threshold_sq = g->thr_sq;
  cfg.origin_at_center = g->ctr;
  cfg.map_vox_num = g->voxel_num;
  cublox::RecenterResult result{};
  cublox::launchRecenter(g->d_occ, g->d_op, g->d_hit, cfg, g->d_slices[0],
                         g->d_slices[1], g->d_slices[2], g->d_result, &result,
                         0);
  CK(cudaGetLastError());
  *action = result.action;
  if (result.action != 0) {
    const int o[3] = {result.new_origin_i.x, result.new_origin_i.y,
                      result.new_origin_i.z};
    set_origin(g, o);
    for (int a = 0; a < 3; ++a) new_origin[a] = o[a];
  }
  return 0;
}

/* planRecenterKernel's device gate alone (no host gate, no clears): runs the
 * reference launcher on a throw-away origin to read back its action.  Used
 * only by the contraction pins.  The map must be large enough that the
 * shift never exceeds half the map. */
int ref_recenter_device_gate(void *hp, const float pos[3], float thr_sq,
                             int *action) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  cublox::RecenterCfg cfg{};
  cfg.pos = make_float3(pos[0], pos[1], pos[2]);
  cfg.origin_f = make_float3(g->origin_f[0], g->origin_f[1], g->origin_f[2]);
  cfg.origin_i = make_int3(g->origin_i[0], g->origin_i[1], g->origin_i[2]);
  cfg.map_size_i = make_int3(g->map[0], g->map[1], g->map[2]);
  cfg.half_map_size_i = make_int3(g->half[0], g->half[1], g->half[2]);
  cfg.resolution = g->res;
  cfg.inv_resolution = g->res_inv;
  cfg.recenter_threshold_sq = thr_sq;
  cfg.origin_at_center = g->ctr;
  cfg.map_vox_num = g->voxel_num;
  cublox::RecenterResult result{};
  cublox::launchRecenter(g->d_occ, g->d_op, g->d_hit, cfg, g->d_slices[0],
                         g->d_slices[1], g->d_slices[2], g->d_result, &result,
                         0);
  CK(cudaGetLastError());
  *action = result.action;
  return 0;
}

static int ensure_fetch(RefGrid *g, int n) {
  if (n <= g->fetch_cap) return 0;
  if (g->d_fstate) CK(cudaFree(g->d_fstate));
  if (g->d_fpos) CK(cudaFree(g->d_fpos));
  if (g->d_fcount) CK(cudaFree(g->d_fcount));
  g->d_fstate = nullptr;
  g->d_fpos = nullptr;
  g->d_fcount = nullptr;
  g->fetch_cap = n;
  CK(cudaMalloc(&g->d_fcount, sizeof(unsigned)));
  CK(cudaMalloc(&g->d_fpos, sizeof(float3) * static_cast<size_t>(n)));
  CK(cudaMalloc(&g->d_fstate, static_cast<size_t>(n)));
  return 0;
}

/* OccupancyGrid::fetchOccupancyAround.  Writes up to out_cap samples in the
 * reference's (atomic, unordered) order.  Returns the sample count or -1. */
int64_t ref_fetch(void *hp, const float center[3], float radius, int filter,
                  int max_results, float *out_pos, unsigned char *out_state,
                  int64_t out_cap) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  if (g->voxel_num <= 0 || radius <= 0.0f) return 0;
  int cg[3];
  for (int a = 0; a < 3; ++a) cg[a] = host_p2g(center[a], g->res_inv, g->ctr);
  float margin = 0.0f;
  {
    const int mx = g->half[0] - std::abs(cg[0] - g->origin_i[0]);
    const int my = g->half[1] - std::abs(cg[1] - g->origin_i[1]);
    if (mx >= 0 && my >= 0) margin = static_cast<float>(std::min(mx, my)) * g->res;
  }
  const float r_eff = std::min(radius, margin);
  if (r_eff <= 0.0f) return 0;
  int gmin[3], gmax[3];
  for (int a = 0; a < 3; ++a) {
    gmin[a] = host_p2g(center[a] - r_eff, g->res_inv, g->ctr);
    gmax[a] = host_p2g(center[a] + r_eff, g->res_inv, g->ctr);
    gmin[a] = std::max(gmin[a], g->origin_i[a] - g->half[a]);
    gmax[a] = std::min(gmax[a], g->origin_i[a] + g->half[a]);
  }
  for (int a = 0; a < 3; ++a)
    if (gmax[a] < gmin[a]) return 0;
  const int disk_r =
      static_cast<int>(std::ceil(static_cast<double>(r_eff * g->res_inv)));
  const int nz = gmax[2] - gmin[2] + 1;
  const int diam = 2 * disk_r + 1;
  const int64_t est = static_cast<int64_t>(diam) * diam * nz;
  if (est <= 0 || est > std::numeric_limits<int>::max()) return 0;
  const unsigned output_cap =
      max_results > 0 ? static_cast<unsigned>(max_results) : 500000u;
  const int fetch_buf =
      static_cast<int>(std::min<int64_t>(output_cap, est));
  if (ensure_fetch(g, fetch_buf)) return -1;
  cublox::OccupancyFetchCfg cfg{};
  cfg.center_g = make_int3(cg[0], cg[1], cg[2]);
  cfg.origin_i = make_int3(g->origin_i[0], g->origin_i[1], g->origin_i[2]);
  cfg.gz_min = gmin[2];
  cfg.gz_max = gmax[2];
  cfg.disk_radius_vox = disk_r;
  cfg.center = make_float3(center[0], center[1], center[2]);
  cfg.radius_sq = r_eff * r_eff;
  cfg.map_size_i = make_int3(g->map[0], g->map[1], g->map[2]);
  cfg.half_map_size_i = make_int3(g->half[0], g->half[1], g->half[2]);
  cfg.resolution = g->res;
  cfg.l_free = g->l_free;
  cfg.l_occupied = g->l_occ;
  cfg.l_unknown = g->l_unknown;
  cfg.origin_at_center = g->ctr;
  cfg.state_filter = filter;
  CK(cudaMemset(g->d_fcount, 0, sizeof(unsigned)));
  const unsigned max_out =
      max_results > 0 ? std::min(static_cast<unsigned>(max_results), output_cap)
                      : output_cap;
  cublox::launchFetchOccupancyAround(cfg, g->d_occ, g->d_fcount, g->d_fpos,
                                     g->d_fstate, output_cap, max_out, 0);
  CK(cudaDeviceSynchronize());
  CK(cudaGetLastError());
  unsigned cnt = 0;
  CK(cudaMemcpy(&cnt, g->d_fcount, sizeof(unsigned), cudaMemcpyDeviceToHost));
  cnt = std::min(cnt, output_cap);
  if (max_results > 0) cnt = std::min(cnt, static_cast<unsigned>(max_results));
  if (cnt == 0) return 0;
  const int64_t n = std::min<int64_t>(cnt, out_cap);
  if (out_pos)
    CK(cudaMemcpy(out_pos, g->d_fpos, sizeof(float3) * n,
                  cudaMemcpyDeviceToHost));
  if (out_state)
    CK(cudaMemcpy(out_state, g->d_fstate, n, cudaMemcpyDeviceToHost));
  return n;
}

int ref_download(void *hp, float *occ, int *op, int *hit) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  const size_t n = static_cast<size_t>(g->voxel_num);
  if (occ) CK(cudaMemcpy(occ, g->d_occ, n * 4, cudaMemcpyDeviceToHost));
  if (op) CK(cudaMemcpy(op, g->d_op, n * 4, cudaMemcpyDeviceToHost));
  if (hit) CK(cudaMemcpy(hit, g->d_hit, n * 4, cudaMemcpyDeviceToHost));
  return 0;
}

int ref_upload(void *hp, const float *occ, const int *op, const int *hit) {
  RefGrid *g = static_cast<RefGrid *>(hp);
  const size_t n = static_cast<size_t>(g->voxel_num);
  if (occ) CK(cudaMemcpy(g->d_occ, occ, n * 4, cudaMemcpyHostToDevice));
  if (op) CK(cudaMemcpy(g->d_op, op, n * 4, cudaMemcpyHostToDevice));
  if (hit) CK(cudaMemcpy(g->d_hit, hit, n * 4, cudaMemcpyHostToDevice));
  return 0;
}

int ref_voxel_num(void *hp) { return static_cast<RefGrid *>(hp)->voxel_num; }

} // extern "C"
