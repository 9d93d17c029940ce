/*
 * cublox CPU oracle — TEST INFRASTRUCTURE ONLY (see cublox_oracle.h).
 *
 * Restates, op by op, the reference's:
 *   index math            include/cublox/utils.cuh:24-176, utils.hpp:24-188
 *   window geometry       src/Grid.cpp:27-92
 *   raycast               src/kernels.cu:33-152
 *   apply                 src/kernels.cu:167-210
 *   update orchestration  src/OccupancyGrid.cpp:181-238
 *   recenter              src/OccupancyGrid.cpp:141-179, kernels.cu:303-499
 *   fetch                 src/OccupancyGrid.cpp:240-356, kernels.cu:506-562
 *   point queries         src/OccupancyGrid.cpp:358-429
 *
 * Build: gcc -O2 -ffp-contract=off (no implicit fusing; fmaf() is explicit).
 */
#include "cublox_oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- float -> int conversions ------------------------------------------ */
/* Device cvt.rzi.s32.f32: saturates, NaN -> 0.                             */
static inline int f2i_dev(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return INT_MAX;
  if (v < -2147483648.0f) return INT_MIN;
  return (int)v;
}
/* x86-64 cvttss2si / cvttsd2si: NaN or out of range -> INT_MIN.             */
static inline int f2i_host(float v) {
  if (v >= -2147483648.0f && v < 2147483648.0f) return (int)v;
  return INT_MIN;
}
static inline int d2i_host(double v) {
  if (v > -2147483649.0 && v < 2147483648.0) return (int)v;
  return INT_MIN;
}
/* Two's-complement int arithmetic as the device does it.                   */
static inline int wadd(int a, int b) { return (int)((unsigned)a + (unsigned)b); }
static inline int wsub(int a, int b) { return (int)((unsigned)a - (unsigned)b); }
static inline int wabs(int a) { return a < 0 ? (int)(0u - (unsigned)a) : a; }

/* ---- sum of squares with a selectable contraction shape ---------------- */
static inline float sos(float x, float y, float z, unsigned shape) {
  switch (shape) {
  case ORC_SOS_FY_FZ:
    return fmaf(z, z, fmaf(y, y, x * x));
  case ORC_SOS_FX_FZ:
    return fmaf(z, z, fmaf(x, x, y * y));
  case ORC_SOS_P_FZ: {
    float s = x * x + y * y;
    return fmaf(z, z, s);
  }
  case ORC_SOS_FY_P: {
    float s = fmaf(y, y, x * x);
    float c = z * z;
    return s + c;
  }
  case ORC_SOS_FX_P: {
    float s = fmaf(x, x, y * y);
    float c = z * z;
    return s + c;
  }
  default: {
    float a = x * x;
    float b = y * y;
    float s = a + b;
    float c = z * z;
    return s + c;
  }
  }
}

/* ---- index math ---------------------------------------------------------- */
int orc_pos_to_global(float p, float res_inv, int origin_at_center, int host,
                      unsigned fp_mode) {
  if (origin_at_center) {
    const float s = p < 0.0f ? -1.0f : 1.0f;
    const float half = s * 0.5f;
    if (host) {
      const float m = p * res_inv;
      return f2i_host(m + half);
    }
    float v;
    if (fp_mode & ORC_FP_CENTER_FMA) {
      v = fmaf(p, res_inv, half);
    } else {
      const float m = p * res_inv;
      v = m + half;
    }
    return f2i_dev(v);
  }
  const float m = p * res_inv;
  return host ? f2i_host(floorf(m)) : f2i_dev(floorf(m));
}

int orc_global_to_local(int g, int map, int half) {
  int l = g % map;
  if (l > half) {
    l -= map;
  } else if (l < -half) {
    l += map;
  }
  return l;
}

int orc_local_to_global(int l, int map, int half, int origin) {
  const int min_g = -half + origin;
  int min_l = min_g % map;
  if (min_l > half) min_l -= map;
  if (min_l < -half) min_l += map;
  int diff = l - min_l;
  if (diff < 0) diff += map;
  return min_g + diff;
}

static inline int hash_local(int lx, int ly, int lz, const int map[3],
                             const int half[3]) {
  return wadd(wadd((int)((unsigned)wadd(lx, half[0]) * (unsigned)map[1] *
                         (unsigned)map[2]),
                   (int)((unsigned)wadd(ly, half[1]) * (unsigned)map[2])),
              wadd(lz, half[2]));
}

int orc_global_to_hash(const int g[3], const int map[3], const int half[3]) {
  return hash_local(orc_global_to_local(g[0], map[0], half[0]),
                    orc_global_to_local(g[1], map[1], half[1]),
                    orc_global_to_local(g[2], map[2], half[2]), map, half);
}

void orc_hash_to_local(int h, const int map[3], const int half[3], int l[3]) {
  const int yz = map[1] * map[2];
  const int x = h / yz;
  const int y = (h - x * yz) / map[2];
  const int z = h - x * yz - y * map[2];
  l[0] = x - half[0];
  l[1] = y - half[1];
  l[2] = z - half[2];
}

float orc_global_to_pos(int g, float res, int origin_at_center) {
  if (origin_at_center) return (float)g * res;
  const float t = (float)g + 0.5f;
  return t * res;
}

float orc_logit(float p) {
  float pc = p;
  const float lo = 1.0e-6f;
  const float hi = 1.0f - 1.0e-6f;
  if (pc < lo) pc = lo;
  if (hi < pc) pc = hi;
  return logf(pc / (1.0f - pc));
}

static inline int in_window(int gx, int gy, int gz, const int o[3],
                            const int h[3]) {
  return wabs(wsub(gx, o[0])) <= h[0] && wabs(wsub(gy, o[1])) <= h[1] &&
         wabs(wsub(gz, o[2])) <= h[2];
}

/* ---- grid lifetime -------------------------------------------------------- */
static void update_origin(orc_grid *g, const int o[3]) {
  for (int a = 0; a < 3; ++a) {
    g->origin_i[a] = o[a];
    g->origin_f[a] = orc_global_to_pos(o[a], g->res, g->origin_at_center);
  }
}

int orc_grid_init(orc_grid *g, const int half[3], float res,
                  int origin_at_center, int has_thr, double thr,
                  const float origin[3]) {
  memset(g, 0, sizeof(*g));
  g->res = res;
  g->res_inv = 1.0f / res;
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    g->half[a] = half[a];
    g->map[a] = 2 * half[a] + 1;
    total *= (int64_t)g->map[a];
  }
  if (total > INT_MAX) return -1;
  g->voxel_num = (int)total;
  g->has_thr = has_thr;
  if (has_thr) {
    g->thr = (float)thr; /* optional<double> -> optional<float> (Grid.hpp:51) */
    g->thr_sq = g->thr * g->thr;
  }
  g->origin_at_center = origin_at_center;
  int o[3];
  for (int a = 0; a < 3; ++a)
    o[a] = orc_pos_to_global(origin[a], g->res_inv, origin_at_center, 1, 0);
  update_origin(g, o);
  g->first_run = 1;
  g->max_range = 25.0f;
  g->l_hit = 0.847f;
  g->l_miss = -0.405f;
  g->l_min = -1.992f;
  g->l_max = 3.476f;
  g->l_free = -0.0004f;
  g->l_occ = 1.7346f;
  g->l_unknown = 0.0f;
  g->fp_mode = ORC_FP_PINNED;
  if (g->voxel_num > 0) {
    g->occ = (float *)calloc((size_t)g->voxel_num, sizeof(float));
    g->op = (int *)calloc((size_t)g->voxel_num, sizeof(int));
    g->hit = (int *)calloc((size_t)g->voxel_num, sizeof(int));
    if (!g->occ || !g->op || !g->hit) {
      orc_grid_free(g);
      return -2;
    }
  }
  return 0;
}

void orc_grid_free(orc_grid *g) {
  free(g->occ);
  free(g->op);
  free(g->hit);
  g->occ = NULL;
  g->op = NULL;
  g->hit = NULL;
}

void orc_grid_reset(orc_grid *g) {
  if (!g->occ) return;
  memset(g->occ, 0, sizeof(float) * (size_t)g->voxel_num);
  memset(g->op, 0, sizeof(int) * (size_t)g->voxel_num);
  memset(g->hit, 0, sizeof(int) * (size_t)g->voxel_num);
  g->first_run = 1;
}

void orc_set_log_odds(orc_grid *g, float l_hit, float l_miss, float l_min,
                      float l_max, float l_free, float l_occ) {
  g->l_hit = l_hit;
  g->l_miss = l_miss;
  g->l_min = l_min;
  g->l_max = l_max;
  g->l_free = l_free;
  g->l_occ = l_occ;
  g->l_unknown = 0.0f;
}

void orc_set_max_range(orc_grid *g, float r) { g->max_range = r; }
void orc_set_fp_mode(orc_grid *g, unsigned mode) { g->fp_mode = mode; }
void orc_set_origin_i(orc_grid *g, const int origin_i[3]) {
  update_origin(g, origin_i);
}

/* ---- raycast ---------------------------------------------------------------- */
typedef struct {
  float o[3];
  int origin_i[3], map[3], half[3];
  float res, inv, max_range;
  int vnum, ctr;
  unsigned fp;
} ray_cfg;

typedef struct {
  int64_t rays, iters, opinc, hitinc;
} ray_acc;

/* One ray.  `op`/`hit` may be NULL (trace only).  Returns 0 when dropped.  */
static int walk(const ray_cfg *c, float ex, float ey, float ez, int *op,
                int *hit, int atomic, int *trace, int cap, int *ntrace,
                ray_acc *acc, int *end_in, int *end_hit) {
  const float ox = c->o[0], oy = c->o[1], oz = c->o[2];
  float dx = ex - ox, dy = ey - oy, dz = ez - oz;
  float L = sqrtf(sos(dx, dy, dz, ORC_FP_RAY_SOS(c->fp)));
  if (L < 1e-6f || !isfinite(L) || !isfinite(ex) || !isfinite(ey) ||
      !isfinite(ez))
    return 0;
  const int clipped = L > c->max_range;
  if (clipped) {
    const float s = c->max_range / L;
    if (c->fp & ORC_FP_CLIP_FMA) {
      ex = fmaf(dx, s, ox);
      ey = fmaf(dy, s, oy);
      ez = fmaf(dz, s, oz);
    } else {
      const float px = dx * s, py = dy * s, pz = dz * s;
      ex = ox + px;
      ey = oy + py;
      ez = oz + pz;
    }
    dx = dx * s;
    dy = dy * s;
    dz = dz * s;
    L = c->max_range;
  }
  const float invL = 1.0f / L;
  const float u[3] = {dx * invL, dy * invL, dz * invL};
  int id[3], end[3], s[3];
  float tD[3], tM[3];
  const float oo[3] = {ox, oy, oz};
  const float ee[3] = {ex, ey, ez};
  for (int a = 0; a < 3; ++a) {
    id[a] = orc_pos_to_global(oo[a], c->inv, c->ctr, 0, c->fp);
    end[a] = orc_pos_to_global(ee[a], c->inv, c->ctr, 0, c->fp);
  }
  for (int a = 0; a < 3; ++a) {
    s[a] = (u[a] > 0) - (u[a] < 0);
    tD[a] = s[a] == 0 ? INFINITY : fabsf(c->res / u[a]);
    float t;
    if (c->ctr) {
      const float hs = 0.5f * (float)s[a];
      t = (float)id[a] + hs;
    } else {
      t = (float)id[a] + (float)(s[a] > 0);
    }
    if (s[a] == 0) {
      tM[a] = INFINITY;
    } else {
      float num;
      if (c->fp & ORC_FP_BOUND_FMA) {
        num = fmaf(t, c->res, -oo[a]);
      } else {
        const float b = t * c->res;
        num = b - oo[a];
      }
      tM[a] = num / u[a];
    }
  }
  const int max_steps =
      wadd(wadd(wadd(wabs(wsub(end[0], id[0])), wabs(wsub(end[1], id[1]))),
                wabs(wsub(end[2], id[2]))),
           4);
  int nt = 0;
  int64_t iters = 0, opinc = 0;
  for (int step = 0; step < max_steps; ++step) {
    if (id[0] == end[0] && id[1] == end[1] && id[2] == end[2]) break;
    ++iters;
    if (in_window(id[0], id[1], id[2], c->origin_i, c->half)) {
      const int h = orc_global_to_hash(id, c->map, c->half);
      if (h >= 0 && h < c->vnum) {
        if (op) {
          if (atomic)
            __atomic_fetch_add(&op[h], 1, __ATOMIC_RELAXED);
          else
            op[h] += 1;
        }
        ++opinc;
        if (trace && nt < cap) trace[nt] = h;
        ++nt;
      }
    }
    if (tM[0] < tM[1]) {
      if (tM[0] < tM[2]) {
        id[0] = wadd(id[0], s[0]);
        tM[0] += tD[0];
      } else {
        id[2] = wadd(id[2], s[2]);
        tM[2] += tD[2];
      }
    } else {
      if (tM[1] < tM[2]) {
        id[1] = wadd(id[1], s[1]);
        tM[1] += tD[1];
      } else {
        id[2] = wadd(id[2], s[2]);
        tM[2] += tD[2];
      }
    }
  }
  int e_in = 0, e_hit = 0;
  if (in_window(end[0], end[1], end[2], c->origin_i, c->half)) {
    const int h = orc_global_to_hash(end, c->map, c->half);
    if (h >= 0 && h < c->vnum) {
      e_in = 1;
      if (op) {
        if (atomic)
          __atomic_fetch_add(&op[h], 1, __ATOMIC_RELAXED);
        else
          op[h] += 1;
      }
      ++opinc;
      if (!clipped) {
        e_hit = 1;
        if (hit) {
          if (atomic)
            __atomic_fetch_add(&hit[h], 1, __ATOMIC_RELAXED);
          else
            hit[h] += 1;
        }
      }
      if (trace && nt < cap) trace[nt] = h;
      ++nt;
    }
  }
  if (ntrace) *ntrace = nt;
  if (end_in) *end_in = e_in;
  if (end_hit) *end_hit = e_hit;
  if (acc) {
    acc->rays += 1;
    acc->iters += iters + 1;
    acc->opinc += opinc;
    acc->hitinc += e_hit;
  }
  return 1;
}

static void make_cfg(const orc_grid *g, const float sensor[3], ray_cfg *c) {
  for (int a = 0; a < 3; ++a) {
    c->o[a] = sensor[a];
    c->origin_i[a] = g->origin_i[a];
    c->map[a] = g->map[a];
    c->half[a] = g->half[a];
  }
  c->res = g->res;
  c->inv = g->res_inv;
  c->max_range = g->max_range;
  c->vnum = g->voxel_num;
  c->ctr = g->origin_at_center;
  c->fp = g->fp_mode;
}

typedef struct {
  const ray_cfg *c;
  const float *x, *y, *z;
  int lo, hi;
  int *op, *hit;
  int atomic;
  ray_acc acc;
} ray_job;

static void *ray_worker(void *arg) {
  ray_job *j = (ray_job *)arg;
  for (int i = j->lo; i < j->hi; ++i)
    walk(j->c, j->x[i], j->y[i], j->z[i], j->op, j->hit, j->atomic, NULL, 0,
         NULL, &j->acc, NULL, NULL);
  return NULL;
}

void orc_raycast(orc_grid *g, const float *x, const float *y, const float *z,
                 int n, const float sensor[3], orc_stats *st, int nthreads) {
  if (n <= 0 || g->voxel_num <= 0) return;
  ray_cfg c;
  make_cfg(g, sensor, &c);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (nthreads > n) nthreads = n;
  ray_job jobs[256];
  pthread_t th[256];
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].c = &c;
    jobs[t].x = x;
    jobs[t].y = y;
    jobs[t].z = z;
    jobs[t].lo = (int)((int64_t)n * t / nthreads);
    jobs[t].hi = (int)((int64_t)n * (t + 1) / nthreads);
    jobs[t].op = g->op;
    jobs[t].hit = g->hit;
    jobs[t].atomic = nthreads > 1;
    memset(&jobs[t].acc, 0, sizeof(ray_acc));
  }
  if (nthreads == 1) {
    ray_worker(&jobs[0]);
  } else {
    for (int t = 0; t < nthreads; ++t)
      pthread_create(&th[t], NULL, ray_worker, &jobs[t]);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  }
  if (st) {
    for (int t = 0; t < nthreads; ++t) {
      st->rays += jobs[t].acc.rays;
      st->voxel_steps += jobs[t].acc.iters;
      st->op_incs += jobs[t].acc.opinc;
      st->hit_incs += jobs[t].acc.hitinc;
    }
  }
}

/* The reference's work units of one scan (kernels.cu:44-137 iterations that
 * did not break, + 1 endpoint per ray that was not dropped).  The loop
 * length does not depend on the window (the window test only decides which
 * iterations increment a counter), so only the binning, the range clip and
 * the contraction pattern enter; no grid is needed. */
int64_t orc_count_steps(float res, int origin_at_center, float max_range, unsigned fp_mode,
                        const float *x, const float *y, const float *z, int n,
                        const float sensor[3], int nthreads) {
  if (n <= 0) return 0;
  ray_cfg c;
  memset(&c, 0, sizeof(c));
  for (int a = 0; a < 3; ++a) {
    c.o[a] = sensor[a];
    c.map[a] = 1;
  }
  c.res = res;
  c.inv = 1.0f / res;
  c.max_range = max_range;
  c.vnum = 1;
  c.ctr = origin_at_center;
  c.fp = fp_mode;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (nthreads > n) nthreads = n;
  ray_job jobs[256];
  pthread_t th[256];
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].c = &c;
    jobs[t].x = x;
    jobs[t].y = y;
    jobs[t].z = z;
    jobs[t].lo = (int)((int64_t)n * t / nthreads);
    jobs[t].hi = (int)((int64_t)n * (t + 1) / nthreads);
    jobs[t].op = NULL;
    jobs[t].hit = NULL;
    jobs[t].atomic = 0;
    memset(&jobs[t].acc, 0, sizeof(ray_acc));
  }
  if (nthreads == 1) {
    ray_worker(&jobs[0]);
  } else {
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, ray_worker, &jobs[t]);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  }
  int64_t steps = 0;
  for (int t = 0; t < nthreads; ++t) steps += jobs[t].acc.iters;
  return steps;
}

/* ---- apply ------------------------------------------------------------------ */
typedef struct {
  orc_grid *g;
  int lo, hi;
  int64_t touched;
} apply_job;

static void *apply_worker(void *arg) {
  apply_job *j = (apply_job *)arg;
  orc_grid *g = j->g;
  const unsigned fp = g->fp_mode;
  int64_t t = 0;
  for (int h = j->lo; h < j->hi; ++h) {
    const int op = g->op[h];
    if (op == 0) continue;
    ++t;
    const int hit = g->hit[h];
    const int miss = op > hit ? op - hit : 0;
    const float s0 = g->occ[h];
    float l = s0 + g->l_unknown;
    if (fp & ORC_FP_MISS_FMA) {
      l = fmaf(g->l_miss, (float)miss, l);
    } else {
      const float p = g->l_miss * (float)miss;
      l = l + p;
    }
    if (fp & ORC_FP_HIT_FMA) {
      l = fmaf(g->l_hit, (float)hit, l);
    } else {
      const float p = g->l_hit * (float)hit;
      l = l + p;
    }
    if (l < g->l_min) l = g->l_min;
    if (l > g->l_max) l = g->l_max;
    g->occ[h] = l - g->l_unknown;
    g->op[h] = 0;
    g->hit[h] = 0;
  }
  j->touched = t;
  return NULL;
}

void orc_apply(orc_grid *g, orc_stats *st, int nthreads) {
  if (g->voxel_num <= 0) return;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  apply_job jobs[256];
  pthread_t th[256];
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].g = g;
    jobs[t].lo = (int)((int64_t)g->voxel_num * t / nthreads);
    jobs[t].hi = (int)((int64_t)g->voxel_num * (t + 1) / nthreads);
    jobs[t].touched = 0;
  }
  if (nthreads == 1) {
    apply_worker(&jobs[0]);
  } else {
    for (int t = 0; t < nthreads; ++t)
      pthread_create(&th[t], NULL, apply_worker, &jobs[t]);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  }
  if (st)
    for (int t = 0; t < nthreads; ++t) st->touched += jobs[t].touched;
}

void orc_update(orc_grid *g, const float *x, const float *y, const float *z,
                int n, const float sensor[3], orc_stats *st, int nthreads) {
  if (g->voxel_num <= 0 || n <= 0) return;
  if (g->first_run) {
    int o[3];
    for (int a = 0; a < 3; ++a)
      o[a] = orc_pos_to_global(sensor[a], g->res_inv, g->origin_at_center, 1,
                               0);
    update_origin(g, o);
    g->first_run = 0;
  }
  orc_raycast(g, x, y, z, n, sensor, st, nthreads);
  orc_apply(g, st, nthreads);
}

int orc_trace_ray(const orc_grid *g, float ex, float ey, float ez,
                  const float sensor[3], int *out, int cap, int *n_total,
                  int *end_in_window, int *end_hit) {
  ray_cfg c;
  make_cfg(g, sensor, &c);
  int nt = 0;
  if (!walk(&c, ex, ey, ez, NULL, NULL, 0, out, cap, &nt, NULL, end_in_window,
            end_hit))
    return -1;
  if (n_total) *n_total = nt;
  return nt < cap ? nt : cap;
}

/* ---- recenter ------------------------------------------------------------- */
static int normalize_slice(int x, int a, int b) {
  const int range = b - a + 1;
  int y = (x - a) % range;
  if (y < 0) y += range;
  return y + a;
}

static void clear_slab(orc_grid *g, int axis, int l) {
  const int *m = g->map, *hf = g->half;
  if (axis == 0) {
    const int base = hash_local(l, -hf[1], -hf[2], m, hf);
    const int n = m[1] * m[2];
    memset(g->occ + base, 0, sizeof(float) * (size_t)n);
    memset(g->op + base, 0, sizeof(int) * (size_t)n);
    memset(g->hit + base, 0, sizeof(int) * (size_t)n);
  } else if (axis == 1) {
    for (int lx = -hf[0]; lx <= hf[0]; ++lx) {
      const int base = hash_local(lx, l, -hf[2], m, hf);
      memset(g->occ + base, 0, sizeof(float) * (size_t)m[2]);
      memset(g->op + base, 0, sizeof(int) * (size_t)m[2]);
      memset(g->hit + base, 0, sizeof(int) * (size_t)m[2]);
    }
  } else {
    for (int lx = -hf[0]; lx <= hf[0]; ++lx)
      for (int ly = -hf[1]; ly <= hf[1]; ++ly) {
        const int h = hash_local(lx, ly, l, m, hf);
        g->occ[h] = 0.0f;
        g->op[h] = 0;
        g->hit[h] = 0;
      }
  }
}

int orc_recenter(orc_grid *g, const float pos[3], int compat, int *host_skip,
                 int new_origin[3], int *slabs[3], int n_slabs[3]) {
  if (host_skip) *host_skip = 0;
  for (int a = 0; a < 3; ++a) {
    if (n_slabs) n_slabs[a] = 0;
    if (new_origin) new_origin[a] = g->origin_i[a];
  }
  if (!g->has_thr || g->voxel_num <= 0) {
    if (host_skip) *host_skip = 1;
    return 0;
  }
  const float dx = pos[0] - g->origin_f[0];
  const float dy = pos[1] - g->origin_f[1];
  const float dz = pos[2] - g->origin_f[2];
  /* Host gate: Eigen squaredNorm, x86-64 without FMA.                      */
  if (sos(dx, dy, dz, ORC_SOS_PLAIN) < g->thr_sq) {
    if (host_skip) *host_skip = 1;
    return 0;
  }
  /* Device re-check in planRecenterKernel.                                 */
  if (sos(dx, dy, dz, ORC_FP_REC_SOS(g->fp_mode)) < g->thr_sq) return 0;
  int no[3], shift[3];
  int max_shift = 0, max_map = 0;
  for (int a = 0; a < 3; ++a) {
    no[a] = orc_pos_to_global(pos[a], g->res_inv, g->origin_at_center, 0,
                              g->fp_mode);
    shift[a] = wsub(no[a], g->origin_i[a]);
    const int as = wabs(shift[a]);
    if (as > max_shift) max_shift = as;
    if (g->map[a] > max_map) max_map = g->map[a];
  }
  if (new_origin)
    for (int a = 0; a < 3; ++a) new_origin[a] = no[a];
  if (max_shift >= max_map) {
    memset(g->occ, 0, sizeof(float) * (size_t)g->voxel_num);
    memset(g->op, 0, sizeof(int) * (size_t)g->voxel_num);
    memset(g->hit, 0, sizeof(int) * (size_t)g->voxel_num);
    update_origin(g, no);
    return 2;
  }
  for (int a = 0; a < 3; ++a) {
    const int sh = shift[a];
    if (sh == 0) continue;
    const int half = g->half[a], map = g->map[a];
    const int min_g = -half + g->origin_i[a];
    const int min_l = min_g % map;
    char *mark = (char *)calloc((size_t)map, 1);
    if (sh > 0) {
      for (int k = 0; k < sh; ++k)
        mark[normalize_slice(min_l + k, -half, half) + half] = 1;
      if (compat)
        for (int k = 0; k < sh; ++k)
          mark[normalize_slice(half - k, -half, half) + half] = 1;
    } else {
      for (int k = -1; k >= sh; --k)
        mark[normalize_slice(min_l + k, -half, half) + half] = 1;
      if (compat)
        for (int k = 0; k < -sh; ++k)
          mark[normalize_slice(-half + k, -half, half) + half] = 1;
    }
    for (int i = 0; i < map; ++i) {
      if (!mark[i]) continue;
      clear_slab(g, a, i - half);
      if (slabs && slabs[a]) slabs[a][n_slabs[a]] = i - half;
      if (n_slabs) n_slabs[a] += 1;
    }
    free(mark);
  }
  update_origin(g, no);
  return 1;
}

/* ---- fetch ---------------------------------------------------------------- */
int64_t orc_fetch(const orc_grid *g, const float center[3], float radius,
                  int filter, int max_results, float *out_pos,
                  uint8_t *out_state, int64_t out_cap, int64_t *n_pass) {
  if (n_pass) *n_pass = 0;
  if (g->voxel_num <= 0 || radius <= 0.0f) return 0;
  /* maxHorizontalInWindowRadius (Grid.cpp:67-78)                           */
  int cg[3];
  for (int a = 0; a < 3; ++a)
    cg[a] = orc_pos_to_global(center[a], g->res_inv, g->origin_at_center, 1, 0);
  float margin = 0.0f;
  {
    const int mx = g->half[0] - wabs(wsub(cg[0], g->origin_i[0]));
    const int my = g->half[1] - wabs(wsub(cg[1], g->origin_i[1]));
    if (mx >= 0 && my >= 0) margin = (float)(mx < my ? mx : my) * g->res;
  }
  const float r_eff = (margin < radius) ? margin : radius; /* std::min */
  if (r_eff <= 0.0f) return 0;
  int gmin[3], gmax[3];
  for (int a = 0; a < 3; ++a) {
    const float lo = center[a] - r_eff;
    const float hi = center[a] + r_eff;
    gmin[a] = orc_pos_to_global(lo, g->res_inv, g->origin_at_center, 1, 0);
    gmax[a] = orc_pos_to_global(hi, g->res_inv, g->origin_at_center, 1, 0);
    const int wmin = g->origin_i[a] - g->half[a];
    const int wmax = g->origin_i[a] + g->half[a];
    if (gmin[a] < wmin) gmin[a] = wmin;
    if (gmax[a] > wmax) gmax[a] = wmax;
  }
  for (int a = 0; a < 3; ++a)
    if (gmax[a] < gmin[a]) return 0;
  const float rv = r_eff * g->res_inv;
  const int disk_r = d2i_host(ceil((double)rv));
  const int gz_min = gmin[2], gz_max = gmax[2];
  const int nz = gz_max - gz_min + 1;
  const int diam = 2 * disk_r + 1;
  const int64_t est = (int64_t)diam * diam * nz;
  if (est <= 0 || est > INT_MAX) return 0;
  const unsigned output_cap =
      max_results > 0 ? (unsigned)max_results : 500000u;
  if (disk_r < 0 || gz_min > gz_max) return 0;
  const float radius_sq = r_eff * r_eff;
  const unsigned fp = g->fp_mode;
  /* Thread extent of the reference launch: ceil(diam/16)*16 per xy axis.    */
  const int ext = ((diam + 15) / 16) * 16;
  int64_t count = 0, written = 0;
  int64_t limit = (int64_t)output_cap;
  if (out_cap < limit) limit = out_cap;
  for (int ix = 0; ix < ext; ++ix) {
    const int gx = cg[0] + (ix - disk_r);
    for (int iy = 0; iy < ext; ++iy) {
      const int gy = cg[1] + (iy - disk_r);
      for (int gz = gz_min; gz <= gz_max; ++gz) {
        if (!in_window(gx, gy, gz, g->origin_i, g->half)) continue;
        const int gg[3] = {gx, gy, gz};
        float p[3], d[3];
        for (int a = 0; a < 3; ++a) {
          const float t =
              g->origin_at_center ? (float)gg[a] : ((float)gg[a] + 0.5f);
          p[a] = t * g->res;
          if (fp & ORC_FP_FETCH_DFMA)
            d[a] = fmaf(t, g->res, -center[a]);
          else
            d[a] = p[a] - center[a];
        }
        if (sos(d[0], d[1], d[2], ORC_FP_FETCH_SOS(fp)) > radius_sq) continue;
        const int h = orc_global_to_hash(gg, g->map, g->half);
        const float l = g->occ[h] + g->l_unknown;
        uint8_t st = 0;
        if (l >= g->l_occ)
          st = 2;
        else if (l < g->l_free)
          st = 1;
        if (filter >= 0 && (int)st != filter) continue;
        ++count;
        if (written < limit) {
          if (out_pos) {
            out_pos[3 * written + 0] = p[0];
            out_pos[3 * written + 1] = p[1];
            out_pos[3 * written + 2] = p[2];
          }
          if (out_state) out_state[written] = st;
          ++written;
        }
      }
    }
  }
  if (n_pass) *n_pass = count;
  return written;
}

/* ---- point queries ------------------------------------------------------- */
int orc_is_state_pos(const orc_grid *g, const float pos[3], int state) {
  int id[3];
  for (int a = 0; a < 3; ++a)
    id[a] = orc_pos_to_global(pos[a], g->res_inv, g->origin_at_center, 1, 0);
  const int inside = in_window(id[0], id[1], id[2], g->origin_i, g->half);
  if (!inside) return state == 0 ? 1 : 0;
  const int h = orc_global_to_hash(id, g->map, g->half);
  float s = 0.0f;
  if (g->occ && h >= 0 && h < g->voxel_num) s = g->occ[h];
  const float l = s + g->l_unknown;
  if (state == 2) return l >= g->l_occ;
  if (state == 1) return l < g->l_free;
  return l >= g->l_free && l < g->l_occ;
}

/* ---- probe search (test infrastructure) ---------------------------------- */
/* Indices of rays whose traced voxel list or endpoint-hit flag differs
 * between two contraction patterns.  Returns how many were written.       */
int orc_find_trace_diff(const orc_grid *g, unsigned mode_a, unsigned mode_b,
                        const float *pts, int n, const float sensor[3],
                        int *out_idx, int cap) {
  ray_cfg ca, cb;
  make_cfg(g, sensor, &ca);
  make_cfg(g, sensor, &cb);
  ca.fp = mode_a;
  cb.fp = mode_b;
  enum { TCAP = 4096 };
  int *ta = (int *)malloc(sizeof(int) * TCAP);
  int *tb = (int *)malloc(sizeof(int) * TCAP);
  int found = 0;
  for (int i = 0; i < n && found < cap; ++i) {
    const float *p = pts + 3 * (size_t)i;
    int na = 0, nb = 0, ia = 0, ib = 0, ha = 0, hb = 0;
    const int ra = walk(&ca, p[0], p[1], p[2], NULL, NULL, 0, ta, TCAP, &na,
                        NULL, &ia, &ha);
    const int rb = walk(&cb, p[0], p[1], p[2], NULL, NULL, 0, tb, TCAP, &nb,
                        NULL, &ib, &hb);
    int diff = ra != rb || na != nb || ia != ib || ha != hb;
    if (!diff) {
      const int m = na < TCAP ? na : TCAP;
      for (int k = 0; k < m; ++k)
        if (ta[k] != tb[k]) {
          diff = 1;
          break;
        }
    }
    if (diff) out_idx[found++] = i;
  }
  free(ta);
  free(tb);
  return found;
}

float orc_sos(float x, float y, float z, unsigned shape) {
  return sos(x, y, z, shape);
}

float orc_fetch_sos(const float c[3], const int gi[3], float res, int ctr,
                    unsigned mode) {
  float d[3];
  for (int a = 0; a < 3; ++a) {
    const float t = ctr ? (float)gi[a] : ((float)gi[a] + 0.5f);
    if (mode & ORC_FP_FETCH_DFMA) {
      d[a] = fmaf(t, res, -c[a]);
    } else {
      const float p = t * res;
      d[a] = p - c[a];
    }
  }
  return sos(d[0], d[1], d[2], ORC_FP_FETCH_SOS(mode));
}

/* main.cpp:666-684, one point at a time. */
int orc_ingest(const float *xyz_aos, int n, const float R[9], const float t[3],
               float max_r2, float *out_aos) {
  int kept = 0;
  if (n > 1000000) n = 1000000; /* kMaxCloudPoints, main.cpp:54, :655-661 */
  for (int i = 0; i < n; ++i) {
    const float x = xyz_aos[3 * i], y = xyz_aos[3 * i + 1], z = xyz_aos[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
    const float r2 = (x * x + y * y) + z * z;  /* squaredNorm */
    if (r2 > max_r2) continue;
    for (int a = 0; a < 3; ++a)
      out_aos[3 * kept + a] = ((R[3 * a] * x + R[3 * a + 1] * y) + R[3 * a + 2] * z) + t[a];
    ++kept;
  }
  return kept;
}

/* depthCallback (main.cpp:596-631): one camera-frame point per pixel,
 * row-major, NaN where the depth is invalid. */
void orc_depth_cloud(const unsigned char *image, int encoding, int width, int height,
                     long long step, const float K[4], float *out_aos) {
  const float nan = NAN;
  for (int v = 0; v < height; ++v) {
    const unsigned char *row = image + (long long)v * step;
    for (int u = 0; u < width; ++u) {
      float *o = out_aos + 3 * ((long long)v * width + u);
      float z;
      int valid;
      if (encoding == 0) {
        unsigned short raw;
        memcpy(&raw, row + 2 * u, 2);
        valid = raw != 0;
        z = (float)raw * 0.001f;
      } else {
        memcpy(&z, row + 4 * u, 4);
        valid = isfinite(z) && z > 0.f;
      }
      if (!valid) {
        o[0] = o[1] = o[2] = nan;
        continue;
      }
      o[0] = ((float)u - K[2]) * z / K[0];
      o[1] = ((float)v - K[3]) * z / K[1];
      o[2] = z;
    }
  }
}

/* publishOccupancyCloudAsync's loop (main.cpp:763-790) with
 * occupancyVizDropBySubsample (:71-84), distanceToOccupancyColor (:275-289)
 * and packRGBFloat (:291-302), on the host's FP32 order. */
static int orc_host_bin(float p, float inv, int ctr) {
  if (ctr) {
    const float s = p < 0.0f ? -1.0f : 1.0f;
    return (int)(p * inv + s * 0.5f);
  }
  return (int)floorf(p * inv);
}

static float orc_clamp01(float v) { return v < 0.f ? 0.f : (1.f < v ? 1.f : v); }

long long orc_viz(const float *pos, long long n, float inv, int ctr, int step, float d_max,
                  long long max_points, const float robot[3], float *out) {
  long long written = 0;
  for (long long i = 0; i < n && written < max_points; ++i) {
    const float *q = pos + 3 * i;
    if (step > 1) {
      const unsigned mix = (unsigned)orc_host_bin(q[0], inv, ctr) ^
                           (unsigned)orc_host_bin(q[1], inv, ctr) ^
                           (unsigned)orc_host_bin(q[2], inv, ctr);
      if (mix % (unsigned)step != 0u) continue;
    }
    const float dx = q[0] - robot[0], dy = q[1] - robot[1], dz = q[2] - robot[2];
    const float d = sqrtf((dx * dx + dy * dy) + dz * dz);
    const float dm = d_max < 1.0f ? 1.0f : d_max;
    const float t = orc_clamp01(d / dm);
    float r, g, b;
    if (t <= 0.5f) {
      const float k = t * 2.0f;
      r = 0.0f; g = 1.0f - k; b = k;
    } else {
      const float k = (t - 0.5f) * 2.0f;
      r = k; g = 0.0f; b = 1.0f - k;
    }
    const unsigned packed = ((unsigned)(orc_clamp01(r) * 255.f) << 16) |
                            ((unsigned)(orc_clamp01(g) * 255.f) << 8) |
                            (unsigned)(orc_clamp01(b) * 255.f);
    float *o = out + 4 * written;
    o[0] = q[0]; o[1] = q[1]; o[2] = q[2];
    memcpy(&o[3], &packed, 4);
    ++written;
  }
  return written;
}
