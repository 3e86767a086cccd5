/* FP64 C restatement of zxtalori's QVM repulsion path.  TEST INFRASTRUCTURE ONLY.
 *
 * The same arithmetic as oracle/qvm.py (pinned against the reference's dense models), in
 * C with OpenMP so that medium sizes finish in seconds: the tests use it as a parity
 * checker and bench.py times it on the host cores as the CPU baseline. The product never
 * links or calls it.
 *
 * Follows: shaders/pairs.wgsl:250-262 (Quey pair), :352-361 (window), :363-416 (near-field
 * membership), shaders/shell.wgsl:18-39 (shell of images near the zone),
 * src/covering.zig:382-396 (zone planes), shaders/relax.wgsl (BB step),
 * shaders/state.wgsl:6-46 (fold), src/pairs.zig:205-215 (mean radius).
 * Quaternions are scalar first, double[4]; symmetry acts on the right.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.14159265358979323846

static void qmul(const double* a, const double* b, double* o) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}
static void normalize(double* a) {
  const double s = 1.0 / sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
  for (int c = 0; c < 4; ++c) a[c] *= s;
}
static double dot4(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

double oracle_mean_radius(double count) {
  const double target = PI * PI / count;
  double lo = 0, hi = PI;
  for (int k = 0; k < 60; ++k) {
    const double m = 0.5 * (lo + hi);
    if (PI * (m - sin(m)) < target) lo = m;
    else hi = m;
  }
  return 0.25 * (lo + hi);
}

/* One Quey pair, optionally windowed (cut_w > 0): force coefficient along the direction,
 * curvature, energy. */
static void quey_pair(const double* x, const double* y, double dm2, double dp2, double cut_z, double cut_w,
                      double* f, double* curv, double* energy) {
  const double nearv = fmax(fmin(dm2, dp2), 1e-30), farv = fmax(fmax(dm2, dp2), 1e-30);
  const double t = sqrt(nearv / farv);
  const double a = fmax(2.0 * atan(t), 1e-12), b = PI - a;
  const double a2 = a * a + 1e-9, b2 = b * b + 1e-9, a3 = a * a * a + 1e-9, b3 = b * b * b + 1e-9;
  const double sine = 2.0 * t / (1.0 + t * t) + 1e-9;
  const double sign = dm2 <= dp2 ? 1.0 : -1.0;
  double d[3] = {x[0] * y[1] - y[0] * x[1] + x[2] * y[3] - x[3] * y[2],
                 x[0] * y[2] - y[0] * x[2] + x[3] * y[1] - x[1] * y[3],
                 x[0] * y[3] - y[0] * x[3] + x[1] * y[2] - x[2] * y[1]};
  double coef = -sign * (b2 - a2) / (a2 * b2 * sine);
  double c = (a3 + b3) / (a3 * b3), e = PI / (a * b);
  if (cut_w > 0) {
    double s = (a - cut_z) * cut_w;
    s = s < 0 ? 0 : (s > 1 ? 1 : s);
    if (s > 0) {
      const double w = 1.0 - s * s * (3.0 - 2.0 * s), slope = -6.0 * s * (1.0 - s) * cut_w;
      coef = w * coef + sign * e * slope / fmax(sin(a), 1e-9);
      c *= w;
      e *= w;
    }
  }
  for (int k = 0; k < 3; ++k) f[k] += coef * d[k];
  *curv += c;
  *energy += e;
}

/* All-pairs force rows (quey_partial semantics). q: n x 4 (normalised here), ops: order x 4.
 * Outputs: force n x 3, curvature, energy, nearest chord^2 and its source (first minimum in
 * (k, j) order). Only the first `count` sources get rows (count <= 0: all), so a bounded
 * sample of a large workload can be timed; with `sources` (count entries), row r belongs
 * to source sources[r] instead. */
void oracle_pair_rows(const double* q_in, int n, const double* ops_in, int order, double* force, double* curv,
                      double* energy, double* nearest, int64_t* nearest_src, int threads, int count,
                      const int64_t* sources) {
  const int rows = (count > 0 && (count < n || sources)) ? count : n;
  double* q = (double*)malloc(sizeof(double) * 4 * n);
  double* img = (double*)malloc(sizeof(double) * 4 * (size_t)n * order);
  memcpy(q, q_in, sizeof(double) * 4 * n);
  for (int i = 0; i < n; ++i) normalize(q + 4 * i);
  for (int k = 0; k < order; ++k)
    for (int j = 0; j < n; ++j) {
      double* y = img + 4 * ((size_t)k * n + j);
      if (k == 0) memcpy(y, q + 4 * j, 32);
      else {
        qmul(q + 4 * j, ops_in + 4 * k, y);
        normalize(y);
      }
    }
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
  for (int r = 0; r < rows; ++r) {
    const int i = sources ? (int)sources[r] : r;
    const double* x = q + 4 * i;
    double f[3] = {0, 0, 0}, c = 0, e = 0, best = 4.0;
    int64_t at = -1;
    for (int k = 0; k < order; ++k)
      for (int j = 0; j < n; ++j) {
        const double* y = img + 4 * ((size_t)k * n + j);
        double dm2 = 0, dp2 = 0;
        for (int t = 0; t < 4; ++t) {
          dm2 += (x[t] - y[t]) * (x[t] - y[t]);
          dp2 += (x[t] + y[t]) * (x[t] + y[t]);
        }
        if (!(j == i && k == 0)) {
          const double m = fmin(dm2, dp2);
          if (m < best) {
            best = m;
            at = j;
          }
        }
        if (j == i) continue;
        quey_pair(x, y, dm2, dp2, 0, 0, f, &c, &e);
      }
    for (int t = 0; t < 3; ++t) force[3 * r + t] = f[t];
    curv[r] = c;
    energy[r] = e;
    nearest[r] = best;
    nearest_src[r] = at;
  }
  free(q);
  free(img);
}

/* ------------------------------------------------------------------ near field */
typedef struct {
  double q[4];
  double p[3];
  int source;
  int identity;
} Site;

static double chart_axis(const double* q, int a) { return q[1 + a] / (1.0 + q[0]); }

/* Near-field rows: every orbit point within S3 angle r = min(1.5, delta d_r) of a source,
 * own orbit excluded from forces, windowed from taper*r (shaders/pairs.wgsl:328-416).
 * Candidate orbit points are the images within the shell of the zone (shell.wgsl:19-39),
 * binned in a grid of the stereographic chart; sources must be zone representatives.
 * Only the first `count` sources get rows (count <= 0: all); with `sources` (count entries),
 * row r belongs to source sources[r] instead. */
void oracle_near_rows(const double* q_in, int n, const double* ops_in, int order, double delta, double taper,
                      double* force, double* curv, double* energy, double* nearest, int64_t* nearest_src,
                      int threads, int count, const int64_t* sources) {
  const int rows = (count > 0 && (count < n || sources)) ? count : n;
  const double r = fmin(1.5, delta * oracle_mean_radius((double)n * order));
  const double cut = pow(2.0 * sin(r / 2.0), 2), chord = 2.0 * sin(r / 2.0);
  const double cut_z = taper * r, cut_w = 1.0 / fmax(1e-9, (1.0 - taper) * r);
  const double margin = sin(r + 1e-4) + 2e-6;
  /* zone planes (src/covering.zig:382-396) */
  const int planes = 2 * order - 1;
  double* plane = (double*)malloc(sizeof(double) * 4 * planes);
  int pc = 0;
  for (int k = 0; k < order; ++k)
    for (int t = 0; t < 2; ++t) {
      const double s = t == 0 ? 1.0 : -1.0;
      if (k == 0 && t == 0) continue;
      double* h = plane + 4 * pc++;
      h[0] = 1.0 - s * ops_in[4 * k];
      for (int c = 1; c < 4; ++c) h[c] = -s * ops_in[4 * k + c];
      normalize(h);
    }
  double* q = (double*)malloc(sizeof(double) * 4 * n);
  memcpy(q, q_in, sizeof(double) * 4 * n);
  for (int i = 0; i < n; ++i) normalize(q + 4 * i);
  /* shell sites */
  int* cnt = (int*)calloc(n + 1, sizeof(int));
  double* gnorm = (double*)malloc(sizeof(double) * 4 * order);
  for (int k = 0; k < order; ++k) {
    memcpy(gnorm + 4 * k, ops_in + 4 * k, 32);
    normalize(gnorm + 4 * k);
  }
#pragma omp parallel for num_threads(threads)
  for (int j = 0; j < n; ++j) {
    const double* o = q + 4 * j;
    int c = 1, rim = 0;
    for (int k = 0; k < planes && !rim; ++k) rim = dot4(o, plane + 4 * k) <= margin;
    if (rim)
      for (int img = 1; img < 2 * order; ++img) {
        double y[4];
        qmul(o, gnorm + 4 * (img / 2), y);
        normalize(y);
        if (img & 1)
          for (int t = 0; t < 4; ++t) y[t] = -y[t];
        int in = y[0] > -0.9999999;
        for (int k = 0; k < planes && in; ++k) in = dot4(y, plane + 4 * k) >= -margin;
        c += in;
      }
    cnt[j + 1] = c;
  }
  for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  const int S = cnt[n];
  Site* site = (Site*)malloc(sizeof(Site) * S);
#pragma omp parallel for num_threads(threads)
  for (int j = 0; j < n; ++j) {
    const double* o = q + 4 * j;
    int at = cnt[j], rim = 0;
    Site* s0 = site + at++;
    memcpy(s0->q, o, 32);
    for (int a = 0; a < 3; ++a) s0->p[a] = chart_axis(o, a);
    s0->source = j;
    s0->identity = 1;
    for (int k = 0; k < planes && !rim; ++k) rim = dot4(o, plane + 4 * k) <= margin;
    if (rim)
      for (int img = 1; img < 2 * order; ++img) {
        double y[4];
        qmul(o, gnorm + 4 * (img / 2), y);
        normalize(y);
        if (img & 1)
          for (int t = 0; t < 4; ++t) y[t] = -y[t];
        int in = y[0] > -0.9999999;
        for (int k = 0; k < planes && in; ++k) in = dot4(y, plane + 4 * k) >= -margin;
        if (!in) continue;
        Site* s = site + at++;
        /* the pair quaternion: the image of the raw source (k=0: the source itself) */
        if (img / 2 == 0) memcpy(s->q, q_in + 4 * j, 32), normalize(s->q);
        else {
          qmul(q_in + 4 * j, ops_in + 4 * (img / 2), s->q);
          normalize(s->q);
        }
        if (img & 1)
          for (int t = 0; t < 4; ++t) s->q[t] = -s->q[t];
        for (int a = 0; a < 3; ++a) s->p[a] = chart_axis(y, a);
        s->source = j;
        s->identity = 0;
      }
  }
  /* chart grid with cells about the chart reach wide */
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int s = 0; s < S; ++s)
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin(lo[a], site[s].p[a]);
      hi[a] = fmax(hi[a], site[s].p[a]);
    }
  double width = 1e-6;
  for (int a = 0; a < 3; ++a) width = fmax(width, hi[a] - lo[a]);
  for (int a = 0; a < 3; ++a) lo[a] -= 0.05 * width;
  width *= 1.1;
  int dim = (int)lround(cbrt(S / 8.0));
  dim = dim < 1 ? 1 : (dim > 128 ? 128 : dim);
  const double per = dim / width;
  int* cell_start = (int*)calloc((size_t)dim * dim * dim + 1, sizeof(int));
  int* cell_of = (int*)malloc(sizeof(int) * S);
  for (int s = 0; s < S; ++s) {
    int c[3];
    for (int a = 0; a < 3; ++a) {
      int v = (int)floor((site[s].p[a] - lo[a]) * per);
      c[a] = v < 0 ? 0 : (v >= dim ? dim - 1 : v);
    }
    cell_of[s] = c[0] + dim * (c[1] + dim * c[2]);
    cell_start[cell_of[s] + 1]++;
  }
  const size_t cells = (size_t)dim * dim * dim;
  for (size_t c = 0; c < cells; ++c) cell_start[c + 1] += cell_start[c];
  int* fill = (int*)malloc(sizeof(int) * cells);
  memcpy(fill, cell_start, sizeof(int) * cells);
  int* order_sites = (int*)malloc(sizeof(int) * S);
  for (int s = 0; s < S; ++s) order_sites[fill[cell_of[s]]++] = s;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
  for (int r = 0; r < rows; ++r) {
    const int i = sources ? (int)sources[r] : r;
    const double* x = q + 4 * i;
    double p[3], f[3] = {0, 0, 0}, c = 0, e = 0, best = 4.0;
    int64_t at = -1;
    for (int a = 0; a < 3; ++a) p[a] = chart_axis(x, a);
    /* chart reach of the cutoff chord (pairs.wgsl:368-378) */
    const double reach = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]), lift = 1.0 + reach * reach;
    double d = 0.5 * chord * lift;
    for (int k = 0; k < 4; ++k) d = 0.5 * chord * sqrt(lift * (1.0 + (reach + d) * (reach + d)));
    if (0.5 * chord * sqrt(lift * (1.0 + (reach + d) * (reach + d))) > d * 1.001) {
      /* no fixed point (wide cutoff): bound |p'| by the chart box's farthest corner */
      double p2 = 0;
      for (int a = 0; a < 3; ++a) {
        const double m = fmax(fabs(lo[a]), fabs(lo[a] + width));
        p2 += m * m;
      }
      d = 0.5 * chord * sqrt(lift * (1.0 + p2));
    }
    d = d * 1.01 + 1e-6;
    int c0[3], c1[3];
    for (int a = 0; a < 3; ++a) {
      int v0 = (int)floor((p[a] - d - lo[a]) * per), v1 = (int)floor((p[a] + d - lo[a]) * per);
      c0[a] = v0 < 0 ? 0 : (v0 >= dim ? dim - 1 : v0);
      c1[a] = v1 < 0 ? 0 : (v1 >= dim ? dim - 1 : v1);
    }
    for (int zc = c0[2]; zc <= c1[2]; ++zc)
      for (int yc = c0[1]; yc <= c1[1]; ++yc) {
        const size_t row = (size_t)dim * (yc + (size_t)dim * zc);
        for (int k = cell_start[row + c0[0]]; k < cell_start[row + c1[0] + 1]; ++k) {
          const Site* s = site + order_sites[k];
          double dm2 = 0;
          for (int t = 0; t < 4; ++t) dm2 += (x[t] - s->q[t]) * (x[t] - s->q[t]);
          if (dm2 > cut) continue;
          if (s->source == i) {
            if (!s->identity && dm2 < best) {
              best = dm2;
              at = i;
            }
            continue;
          }
          if (dm2 < best || (dm2 == best && s->source < at)) {
            best = dm2;
            at = s->source;
          }
          double dp2 = 0;
          for (int t = 0; t < 4; ++t) dp2 += (x[t] + s->q[t]) * (x[t] + s->q[t]);
          quey_pair(x, s->q, dm2, dp2, cut_z, cut_w, f, &c, &e);
        }
      }
    for (int t = 0; t < 3; ++t) force[3 * r + t] = f[t];
    curv[r] = c;
    energy[r] = e;
    nearest[r] = best;
    nearest_src[r] = at;
  }
  free(plane);
  free(q);
  free(cnt);
  free(gnorm);
  free(site);
  free(cell_start);
  free(cell_of);
  free(fill);
  free(order_sites);
}
