/*
 * Seeded synthetic DDM movies: the oracle's restatement of
 * motility-ddm/test/sim.mjs (mulberry32, Marsaglia polar normals,
 * Marsaglia-Tsang gammas, periodic Gaussian blobs, 8-bit quantisation, drop
 * masks) and of ddm_ref.js shuffleOrder. The RNG streams are consumed in the
 * reference's order so the same seed gives the same movie.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
  uint32_t a;
  int has_spare;
  double spare;
} rng_t;

/* mulberry32 (sim.mjs:14-23): 32-bit wrap-around arithmetic throughout. */
static double rng_uniform(rng_t *r) {
  r->a = r->a + 0x6d2b79f5u;
  uint32_t t = r->a;
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  return (double)(t ^ (t >> 14)) / 4294967296.0;
}

static void rng_init(rng_t *r, uint32_t seed) {
  r->a = seed;
  r->has_spare = 0;
  r->spare = 0;
}

/* Marsaglia polar method with a cached spare (sim.mjs:29-44). */
static double rng_normal(rng_t *r) {
  if (r->has_spare) {
    r->has_spare = 0;
    return r->spare;
  }
  double x, y, s;
  do {
    x = 2 * rng_uniform(r) - 1;
    y = 2 * rng_uniform(r) - 1;
    s = x * x + y * y;
  } while (s >= 1 || s == 0);
  const double f = sqrt((-2 * log(s)) / s);
  r->spare = y * f;
  r->has_spare = 1;
  return x * f;
}

/* Gamma(k, theta), Marsaglia-Tsang (sim.mjs:46-61). */
static double rng_gamma(rng_t *r, double k, double theta) {
  if (k < 1) return rng_gamma(r, k + 1, theta) * pow(rng_uniform(r), 1 / k);
  const double d = k - 1.0 / 3;
  const double c = 1 / sqrt(9 * d);
  for (;;) {
    double x, v;
    do {
      x = rng_normal(r);
      v = 1 + c * x;
    } while (v <= 0);
    v = v * v * v;
    const double uu = rng_uniform(r);
    if (uu < 1 - 0.0331 * pow(x, 4)) return d * v * theta;
    if (log(uu) < 0.5 * x * x + d * (1 - v + log(v))) return d * v * theta;
  }
}

void or_mulberry32(uint32_t seed, double *out, int n) {
  rng_t r;
  rng_init(&r, seed);
  for (int i = 0; i < n; i++) out[i] = rng_uniform(&r);
}

void or_rng_normals(uint32_t seed, double *out, int n) {
  rng_t r;
  rng_init(&r, seed);
  for (int i = 0; i < n; i++) out[i] = rng_normal(&r);
}

void or_rng_gammas(uint32_t seed, double k, double theta, double *out, int n) {
  rng_t r;
  rng_init(&r, seed);
  for (int i = 0; i < n; i++) out[i] = rng_gamma(&r, k, theta);
}

static double js_round(double x) {
  const double f = floor(x);
  return (x - f >= 0.5) ? f + 1.0 : f;
}

typedef struct {
  double x, y, vx, vy;
  int mobile;
} particle;

/* Render a movie (sim.mjs:90-186). */
void or_simulate(const or_sim_params *p, uint8_t *frames, uint8_t *valid,
                 double *truth) {
  const int N = p->N, T = p->T;
  const double dt = 1 / p->fps, dxUm = p->dxUm;
  rng_t rng;
  rng_init(&rng, p->seed);
  const double sig = p->blobSigmaPx, amp = p->amp, bg = p->background;
  const double noise = p->noise, D = p->Dum2s;
  const double Lf = N * dxUm;
  double Vx = 0, Vy = 0;
  if (p->hasDrift) {
    Vx = p->driftSpeed * cos((p->driftAngleDeg * M_PI) / 180);
    Vy = p->driftSpeed * sin((p->driftAngleDeg * M_PI) / 180);
  }
  const int np = p->nSwim + p->nPassive + p->nFixed;
  particle *parts = (particle *)calloc(np > 0 ? np : 1, sizeof(particle));
  int cnt = 0;
  double speedSum = 0;
  if (p->nSwim > 0) {
    const double Z = pow(p->swimVbar / p->swimSigma, 2) - 1;
    for (int i = 0; i < p->nSwim; i++) {
      const double v = rng_gamma(&rng, Z + 1, p->swimVbar / (Z + 1));
      speedSum += v;
      const double phi = 2 * M_PI * rng_uniform(&rng);
      double s = 1;
      if (!p->swim2d) {
        const double cz = 2 * rng_uniform(&rng) - 1;
        s = sqrt(1 - cz * cz);
      }
      particle q;
      q.x = rng_uniform(&rng) * Lf;
      q.y = rng_uniform(&rng) * Lf;
      q.vx = v * s * cos(phi);
      q.vy = v * s * sin(phi);
      q.mobile = 1;
      parts[cnt++] = q;
    }
  }
  for (int i = 0; i < p->nPassive; i++) {
    particle q = {0, 0, 0, 0, 1};
    q.x = rng_uniform(&rng) * Lf;
    q.y = rng_uniform(&rng) * Lf;
    parts[cnt++] = q;
  }
  for (int i = 0; i < p->nFixed; i++) {
    particle q = {0, 0, 0, 0, 0};
    q.x = rng_uniform(&rng) * Lf;
    q.y = rng_uniform(&rng) * Lf;
    parts[cnt++] = q;
  }
  const int R = (int)ceil(4 * sig);
  const int S = 2 * R + 2;
  double *gx = (double *)malloc(sizeof(double) * S);
  double *gy = (double *)malloc(sizeof(double) * S);
  double *img = (double *)malloc(sizeof(double) * N * N);
  const double step = sqrt(2 * D * dt);
  for (int t = 0; t < T; t++) {
    for (int i = 0; i < N * N; i++) img[i] = bg;
    for (int k = 0; k < np; k++) {
      const particle *q = &parts[k];
      const double px = q->x / dxUm, py = q->y / dxUm;
      const int x0 = (int)floor(px) - R, y0 = (int)floor(py) - R;
      for (int i = 0; i < S; i++) {
        const double ddx = x0 + i - px, ddy = y0 + i - py;
        gx[i] = exp((-ddx * ddx) / (2 * sig * sig));
        gy[i] = amp * exp((-ddy * ddy) / (2 * sig * sig));
      }
      for (int j = 0; j < S; j++) {
        const int yy = (((y0 + j) % N) + N) % N;
        const double gyj = gy[j];
        double *row = img + (size_t)yy * N;
        for (int i = 0; i < S; i++) {
          const int xx = (((x0 + i) % N) + N) % N;
          row[xx] += gx[i] * gyj;
        }
      }
    }
    uint8_t *f = frames + (size_t)t * N * N;
    for (int i = 0; i < N * N; i++) {
      const double v = js_round((img[i] + noise * rng_normal(&rng)) * 255);
      f[i] = v < 0 ? 0 : v > 255 ? 255 : (uint8_t)v;
    }
    for (int k = 0; k < np; k++) {
      particle *q = &parts[k];
      if (!q->mobile) continue;
      q->x += (q->vx + Vx) * dt + step * rng_normal(&rng);
      q->y += (q->vy + Vy) * dt + step * rng_normal(&rng);
      q->x = fmod(fmod(q->x, Lf) + Lf, Lf);
      q->y = fmod(fmod(q->y, Lf) + Lf, Lf);
    }
  }
  for (int t = 0; t < T; t++) valid[t] = 1;
  rng_t drng;
  rng_init(&drng, p->seed * 7919u + 13u);
  if (p->dropExact) {
    int *idx = (int *)malloc(sizeof(int) * (T - 1));
    for (int i = 0; i < T - 1; i++) idx[i] = i + 1;
    for (int i = T - 2; i > 0; i--) {
      const int j = (int)floor(rng_uniform(&drng) * (i + 1));
      const int tmp = idx[i];
      idx[i] = idx[j];
      idx[j] = tmp;
    }
    for (int i = 0; i < p->dropExact; i++) valid[idx[i]] = 0;
    free(idx);
  } else if (p->dropFrac > 0) {
    for (int t = 1; t < T; t++)
      if (rng_uniform(&drng) < p->dropFrac) valid[t] = 0;
  }
  if (truth) {
    truth[0] = p->nSwim > 0 ? speedSum / p->nSwim : 0;
    truth[1] = Vx;
    truth[2] = Vy;
    truth[3] = D;
  }
  free(parts);
  free(gx);
  free(gy);
  free(img);
}

/* Control-1 shuffle of (slot, mask) pairs (ddm_ref.js:510-519). */
void or_shuffle_order(uint32_t *order, double *mask, int T, uint32_t seed) {
  rng_t r;
  rng_init(&r, seed);
  for (int i = T - 1; i > 0; i--) {
    const int j = (int)floor(rng_uniform(&r) * (i + 1));
    const uint32_t to = order[i];
    order[i] = order[j];
    order[j] = to;
    const double tm = mask[i];
    mask[i] = mask[j];
    mask[j] = tm;
  }
}
