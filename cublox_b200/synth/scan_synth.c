/*
 * Synthetic LiDAR scene ray caster (input generation for tests and bench).
 *
 * The scene is the ground plane z = 0 plus axis-aligned boxes.  Each ray
 * returns the distance to the nearest surface (or +inf).  Boxes are binned by
 * the azimuth interval their footprint subtends from the sensor, so a ray only
 * tests the boxes of its own azimuth bin.  Double precision throughout; the
 * caller rounds the resulting points to float32.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define NBINS 720

typedef struct {
  const double *o;
  const double *dirs;
  const double *boxes;
  int lo, hi;
  int ground;
  const int *bin_start;
  const int *bin_items;
  double *out;
} job_t;

static double hit_box(const double o[3], const double d[3], const double *b) {
  double t0 = 0.0, t1 = INFINITY;
  for (int a = 0; a < 3; ++a) {
    const double lo = b[a], hi = b[a + 3];
    if (fabs(d[a]) < 1e-15) {
      if (o[a] < lo || o[a] > hi) return INFINITY;
      continue;
    }
    double ta = (lo - o[a]) / d[a];
    double tb = (hi - o[a]) / d[a];
    if (ta > tb) {
      const double t = ta;
      ta = tb;
      tb = t;
    }
    if (ta > t0) t0 = ta;
    if (tb < t1) t1 = tb;
    if (t0 > t1) return INFINITY;
  }
  return t0 > 1e-9 ? t0 : INFINITY;
}

static int az_bin(double ang) {
  double u = (ang + M_PI) / (2.0 * M_PI) * NBINS;
  int b = (int)floor(u);
  b %= NBINS;
  if (b < 0) b += NBINS;
  return b;
}

static void *worker(void *arg) {
  job_t *j = (job_t *)arg;
  for (int i = j->lo; i < j->hi; ++i) {
    const double *d = j->dirs + 3 * (size_t)i;
    double best = INFINITY;
    if (j->ground && d[2] < 0.0) {
      const double t = -j->o[2] / d[2];
      if (t > 1e-9) best = t;
    }
    const int b = az_bin(atan2(d[1], d[0]));
    for (int k = j->bin_start[b]; k < j->bin_start[b + 1]; ++k) {
      const double t = hit_box(j->o, d, j->boxes + 6 * (size_t)j->bin_items[k]);
      if (t < best) best = t;
    }
    j->out[i] = best;
  }
  return NULL;
}

/* Returns 0 on success. */
int synth_cast(const double o[3], const double *dirs, int n,
               const double *boxes, int nb, int ground, double *out_t,
               int nthreads) {
  /* azimuth interval of every box footprint, as bins [b0, b1] (wrapping) */
  int *b0 = (int *)malloc(sizeof(int) * (size_t)(nb > 0 ? nb : 1));
  int *b1 = (int *)malloc(sizeof(int) * (size_t)(nb > 0 ? nb : 1));
  int *count = (int *)calloc(NBINS + 1, sizeof(int));
  if (!b0 || !b1 || !count) return -1;
  for (int k = 0; k < nb; ++k) {
    const double *b = boxes + 6 * (size_t)k;
    if (o[0] >= b[0] && o[0] <= b[3] && o[1] >= b[1] && o[1] <= b[4]) {
      b0[k] = 0;
      b1[k] = NBINS - 1;
    } else {
      const double cx = 0.5 * (b[0] + b[3]) - o[0];
      const double cy = 0.5 * (b[1] + b[4]) - o[1];
      const double ca = atan2(cy, cx);
      double lo = 0.0, hi = 0.0;
      for (int c = 0; c < 4; ++c) {
        const double px = (c & 1 ? b[3] : b[0]) - o[0];
        const double py = (c & 2 ? b[4] : b[1]) - o[1];
        double da = atan2(py, px) - ca;
        while (da > M_PI) da -= 2.0 * M_PI;
        while (da < -M_PI) da += 2.0 * M_PI;
        if (da < lo) lo = da;
        if (da > hi) hi = da;
      }
      const int s = az_bin(ca + lo) - 1;
      const int e = az_bin(ca + hi) + 1;
      b0[k] = s;
      b1[k] = e < s ? e + NBINS : e;
      if (b1[k] - b0[k] >= NBINS) {
        b0[k] = 0;
        b1[k] = NBINS - 1;
      }
    }
    for (int q = b0[k]; q <= b1[k]; ++q) count[((q % NBINS) + NBINS) % NBINS]++;
  }
  int *start = (int *)calloc(NBINS + 1, sizeof(int));
  for (int q = 0; q < NBINS; ++q) start[q + 1] = start[q] + count[q];
  int *items = (int *)malloc(sizeof(int) * (size_t)(start[NBINS] + 1));
  int *fill = (int *)calloc(NBINS, sizeof(int));
  for (int k = 0; k < nb; ++k)
    for (int q = b0[k]; q <= b1[k]; ++q) {
      const int qq = ((q % NBINS) + NBINS) % NBINS;
      items[start[qq] + fill[qq]++] = k;
    }
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 64) nthreads = 64;
  if (nthreads > n) nthreads = n > 0 ? n : 1;
  job_t jobs[64];
  pthread_t th[64];
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].o = o;
    jobs[t].dirs = dirs;
    jobs[t].boxes = boxes;
    jobs[t].lo = (int)((long long)n * t / nthreads);
    jobs[t].hi = (int)((long long)n * (t + 1) / nthreads);
    jobs[t].ground = ground;
    jobs[t].bin_start = start;
    jobs[t].bin_items = items;
    jobs[t].out = out_t;
  }
  if (nthreads == 1) {
    worker(&jobs[0]);
  } else {
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, worker, &jobs[t]);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  }
  free(b0);
  free(b1);
  free(count);
  free(start);
  free(items);
  free(fill);
  return 0;
}
