/* ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of the reference's ray tracer (flyverse/world.py:20-43 value noise,
 * :162-211 intersection, :264-300 shading and patterns; flyverse/batch_world.py:94-147 for one
 * scene per row; flyverse/batch_sim.py:192-201 for the eye's pose turn and column sums), written
 * the way the reference evaluates it: every primitive class reduced to its nearest hit, classes
 * compared in order, the shadow ray's nearest hit over all primitives compared with the light
 * distance. Float32 throughout, each operation rounded on its own (built with -ffp-contract=off);
 * the vector length is the fused multiply-add chain the reference's CPU norm uses.
 * Reads the same argument record as the CUDA kernel (flyb_trace_args), on host pointers.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "../include/flyb200.h"

#define INF_T 1e9f
#define EPS_T 1e-4f
#define TINY 1e-9f

static float len3(float x, float y, float z) { return sqrtf(fmaf(z, z, fmaf(y, y, x * x))); }

static float rem_floor(float a, float b) {  /* torch.remainder for floats */
  float r = fmodf(a, b);
  if (r != 0.f && ((r < 0.f) != (b < 0.f))) r += b;
  return r;
}

static long long pymod64(long long a, long long m) {
  long long r = a % m;
  return r < 0 ? r + m : r;
}

static float hash3(long long x, long long y, long long z) {
  /* int64 arithmetic that wraps like torch's */
  uint64_t lin = (uint64_t)x * 374761393ull + (uint64_t)y * 668265263ull + (uint64_t)z * 2147483647ull;
  long long h = pymod64((long long)lin, 2147483647ll);
  h = pymod64((long long)((uint64_t)(h ^ (h >> 13)) * 1274126177ull), 2147483647ll);
  return (float)(h % 65536) / 32768.0f - 1.0f;
}

static float noise(const float p[3], float scale) {
  float q[3], f[3];
  long long i[3];
  for (int c = 0; c < 3; ++c) {
    q[c] = p[c] / scale;
    i[c] = (long long)floorf(q[c]);
    f[c] = q[c] - (float)i[c];
    f[c] = f[c] * f[c] * (3.f - 2.f * f[c]);
  }
  float out = 0.f;
  for (int corner = 0; corner < 8; ++corner) {
    const int dx = corner >> 2, dy = (corner >> 1) & 1, dz = corner & 1;
    const float wx = dx ? f[0] : 1.f - f[0], wy = dy ? f[1] : 1.f - f[1], wz = dz ? f[2] : 1.f - f[2];
    out += wx * wy * wz * hash3(i[0] + dx, i[1] + dy, i[2] + dz);
  }
  return out;
}

typedef struct {
  int ns, nb, np;
  const float *sph, *box, *pln, *mat, *light;
} scene_t;

typedef struct {
  float t, n[3];
  int id;
} hit_t;

static hit_t intersect(const scene_t* s, const float o[3], const float d[3]) {
  hit_t h = {INF_T, {0.f, 0.f, 0.f}, s->ns + s->nb + s->np};
  if (s->ns) {
    float tmin = INF_T;
    int si = 0;
    for (int k = 0; k < s->ns; ++k) {
      const float* sp = s->sph + 6 * k;
      float oc[3], dd[3];
      for (int c = 0; c < 3; ++c) oc[c] = (o[c] - sp[c]) / sp[3 + c], dd[c] = d[c] / sp[3 + c];
      const float a = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
      const float b = 2 * (oc[0] * dd[0] + oc[1] * dd[1] + oc[2] * dd[2]);
      const float cc = (oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2]) - 1;
      const float disc = b * b - 4 * a * cc;
      const float sq = sqrtf(disc > 0.f ? disc : 0.f);
      const float t0 = (-b - sq) / (2 * a), t1 = (-b + sq) / (2 * a);
      float t = t0 > EPS_T ? t0 : t1;
      t = (disc > 0.f && t > EPS_T) ? t : INF_T;
      if (t < tmin) tmin = t, si = k;
    }
    if (tmin < h.t) {
      const float* sp = s->sph + 6 * si;
      float n[3];
      for (int c = 0; c < 3; ++c) n[c] = (o[c] + d[c] * tmin - sp[c]) / (sp[3 + c] * sp[3 + c]);
      float l = len3(n[0], n[1], n[2]);
      if (l < TINY) l = TINY;
      h.t = tmin, h.id = si;
      for (int c = 0; c < 3; ++c) h.n[c] = n[c] / l;
    }
  }
  if (s->nb) {
    float inv[3];
    for (int c = 0; c < 3; ++c) inv[c] = 1.0f / (fabsf(d[c]) < TINY ? TINY : d[c]);
    float tmin = INF_T;
    int bi = 0, axis = 0;
    for (int k = 0; k < s->nb; ++k) {
      const float* bx = s->box + 6 * k;
      float tn[3], tf[3];
      for (int c = 0; c < 3; ++c) {
        const float lo = (bx[c] - o[c]) * inv[c], hi = (bx[3 + c] - o[c]) * inv[c];
        tn[c] = lo < hi ? lo : hi;
        tf[c] = lo > hi ? lo : hi;
      }
      int ax = 0;
      float enter = tn[0];
      for (int c = 1; c < 3; ++c)
        if (tn[c] > enter) enter = tn[c], ax = c;
      float leave = tf[0];
      for (int c = 1; c < 3; ++c)
        if (tf[c] < leave) leave = tf[c];
      const float t = (leave > enter && enter > EPS_T) ? enter : INF_T;
      if (t < tmin) tmin = t, bi = k, axis = ax;
    }
    if (tmin < h.t) {
      const float sgn = d[axis] > 0.f ? 1.f : (d[axis] < 0.f ? -1.f : 0.f);
      h.t = tmin, h.id = s->ns + bi;
      for (int c = 0; c < 3; ++c) h.n[c] = c == axis ? -sgn : 0.f;
    }
  }
  if (s->np) {
    float tmin = INF_T;
    int pi = 0;
    for (int k = 0; k < s->np; ++k) {
      const float* pl = s->pln + 6 * k;
      const float denom = d[0] * pl[3] + d[1] * pl[4] + d[2] * pl[5];
      const float num = (pl[0] - o[0]) * pl[3] + (pl[1] - o[1]) * pl[4] + (pl[2] - o[2]) * pl[5];
      float t = num / (fabsf(denom) < TINY ? TINY : denom);
      t = (t > EPS_T && fabsf(denom) > TINY) ? t : INF_T;
      if (t < tmin) tmin = t, pi = k;
    }
    if (tmin < h.t) {
      const float* pn = s->pln + 6 * pi + 3;
      const float facing = pn[0] * d[0] + pn[1] * d[1] + pn[2] * d[2];
      h.t = tmin, h.id = s->ns + s->nb + pi;
      for (int c = 0; c < 3; ++c) h.n[c] = facing > 0.f ? -pn[c] : pn[c];
    }
  }
  return h;
}

static void trace_one(const scene_t* s, float detail, const float o[3], const float d[3], float out[4]) {
  const hit_t h = intersect(s, o, d);
  if (!(h.t < INF_T)) {
    out[0] = out[1] = out[2] = out[3] = 0.f;
    return;
  }
  float p[3], tl[3], l[3], so[3];
  for (int c = 0; c < 3; ++c) p[c] = o[c] + d[c] * h.t, tl[c] = s->light[c] - p[c];
  const float dist = len3(tl[0], tl[1], tl[2]);
  const float dc = dist < TINY ? TINY : dist;
  for (int c = 0; c < 3; ++c) l[c] = tl[c] / dc;
  float lam = h.n[0] * l[0] + h.n[1] * l[1] + h.n[2] * l[2];
  if (lam < 0.f) lam = 0.f;
  for (int c = 0; c < 3; ++c) so[c] = p[c] + h.n[c] * 1e-3f;
  const hit_t sh = intersect(s, so, l);
  const float lit = sh.t >= dist ? 1.f : 0.f;
  const float falloff = 4.0f / (1.0f + dist * dist);
  const float* m = s->mat + 16 * h.id;
  const int pat = (int)m[13];
  const float sc = m[12];
  const float fx = floorf(p[0] / sc), fy = floorf(p[1] / sc);
  const int checks = rem_floor(fx + fy, 2) == 1;
  const float horiz = fabsf(h.n[0]) > 0.5f ? fy : fx;
  const int stripes = rem_floor(horiz, 2) == 1;
  const int planks = rem_floor(fy, 2) == 1 || rem_floor(fx + 3 * fy, 7) == 0;
  const int second = pat == 1 ? checks : (pat == 2 ? stripes : (pat == 3 ? planks : 0));
  float refl[4];
  for (int c = 0; c < 4; ++c) refl[c] = second ? m[4 + c] : m[c];
  if (detail > 0) {
    float mm = 1.0f + detail * (0.5f * noise(p, 0.02f) + 0.3f * noise(p, 0.008f) + 0.2f * noise(p, 0.003f));
    if (mm < 0.1f) mm = 0.1f;
    for (int c = 0; c < 4; ++c) refl[c] = refl[c] * mm;
  }
  const float shine = lam * lit * falloff;
  for (int c = 0; c < 4; ++c) out[c] = refl[c] * (s->light[7 + c] + s->light[3 + c] * shine) + m[8 + c];
}

int oracle_trace(const flyb_trace_args* a, int threads) {
  if (!a || a->samples < 1 || a->rays % a->samples) return 1;
  const int objects = a->n_sph + a->n_box + a->n_pln;
  const int floats = 6 * objects + 16 * (objects + 1) + 12;
  const int outputs = a->rays / a->samples;
  const long long total = (long long)a->batch * outputs;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
  for (long long u = 0; u < total; ++u) {
    const int b = (int)(u / outputs), col = (int)(u % outputs);
    scene_t s;
    s.ns = a->n_sph, s.nb = a->n_box, s.np = a->n_pln;
    s.sph = a->scene + (size_t)b * floats;
    s.box = s.sph + 6 * s.ns;
    s.pln = s.box + 6 * s.nb;
    s.mat = s.pln + 6 * s.np;
    s.light = s.mat + 16 * (objects + 1);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int j = 0; j < a->samples; ++j) {
      const long long ray = (long long)col * a->samples + j;
      float o[3], d[3], rad[4];
      for (int c = 0; c < 3; ++c) {
        o[c] = a->shared_origin ? a->origins[3 * b + c] : a->origins[3 * ((size_t)b * a->rays + ray) + c];
        if (a->pose) {
          const double* e = a->eye_dirs + 3 * ray;
          const double* P = a->pose + 9 * b;
          d[c] = (float)(e[0] * P[c] + e[1] * P[3 + c] + e[2] * P[6 + c]);
        } else {
          d[c] = a->dirs[3 * ((size_t)b * a->rays + ray) + c];
        }
      }
      trace_one(&s, a->detail, o, d, rad);
      if (a->samples == 1) {
        for (int c = 0; c < 4; ++c) acc[c] = rad[c];
      } else {
        for (int c = 0; c < 4; ++c) acc[c] = acc[c] + rad[c] * a->weights[j];
      }
    }
    for (int c = 0; c < 4; ++c) a->out[4 * (size_t)u + c] = acc[c];
  }
  return 0;
}
