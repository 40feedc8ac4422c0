/*
 * flyb200 ORACLE -- test infrastructure only. Nothing in the product links or calls this file;
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm use it as the
 * checker and as the timed CPU port.
 *
 * A plain-C restatement of the reference's per-step brain update:
 *
 *  - oracle_lif_run: the LIF step of flyverse/brain.py:_step_inference (brain.py:829-870), in the
 *    order of operations of that loop and of flyverse/kernels/neural.cu:18-52, with the synaptic
 *    input delivered through an exact delay ring instead of the float spike buffer
 *    (brain.py:485-487, 833, 858-865). Ring slot r holds the input due at the step that reads it;
 *    a spike of step t is added to slot (pos(t) + D) mod R, so the delay is exactly D steps as in
 *    the reference buffer. COUNT rings sum signed integer synapse counts (exact), FIXED rings sum
 *    per-edge Q32.32 millivolts (each edge rounded once, then an exact integer sum), so both are
 *    independent of summation order.
 *  - Poisson uniforms come either from a caller array (parity mode: the reference's torch CPU
 *    generator draws, brain.py:848) or from Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
 *    "Parallel random numbers: as easy as 1, 2, 3", SC'11), restated from the paper.
 *  - oracle_optic_run: the optic substep of flyverse/optic.py:_substep (optic.py:525-551) and of
 *    neural.cu:62-79 in FP32 with the reference's addition order, or in FP64.
 *  - oracle_spmm: the held-input products of optic.py:579-580, 599-602.
 *
 * All float arithmetic is written one IEEE operation per statement; build with
 * -ffp-contract=off so that no multiply-add is contracted (the reference builds its CUDA
 * kernels with --fmad=false, flyverse/cuda.py:51).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/flyb200.h"

/* ------------------------------------------------------------------ Philox4x32-10 */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += W0; k1 += W1; }
    uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}

/* Uniform in [0, 1) with 24 random bits, for (seed, step, neuron, fly). */
float oracle_uniform(uint64_t seed, uint64_t step, uint32_t neuron, uint32_t fly) {
  uint32_t c[4] = {(uint32_t)step, (uint32_t)(step >> 32), neuron, fly};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return (float)(c[0] >> 8) * (1.0f / 16777216.0f);
}

void oracle_philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t* out) {
  uint32_t c[4] = {c0, c1, c2, c3};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  memcpy(out, c, sizeof c);
}

/* ------------------------------------------------------------------ LIF */
#define Q32 4294967296.0

static inline int64_t fixed_of(float w, float x) {
  /* w and x are float32: their product is exact in double, the scaling by 2^32 too;
   * llrint rounds half to even, like the device's __double2ll_rn. */
  return (int64_t)llrint((double)w * (double)x * Q32);
}

static inline float float_of_fixed(int64_t acc) {
  return (float)((double)acc * (1.0 / Q32));
}

/* One fly, one step. Returns the synaptic events this fly delivered. */
static uint64_t lif_fly_step(const flyb_lif_args* a, int b, int k, const float* P, unsigned char* fired_out,
                             long long step0, int ring_pos) {
  const int n = a->n, B = a->batch, R = a->ring_slots;
  const int rs = (int)(((long long)ring_pos + k) % R);
  const int ws = (int)(((long long)ring_pos + k + a->n_delay) % R);
  const long long step = step0 + k;
  const int flags = a->flags;
  const float v_rest = P[FLYB_P_V_REST], v_reset = P[FLYB_P_V_RESET], v_th = P[FLYB_P_V_TH];
  const float a_m = P[FLYB_P_A_M], a_s = P[FLYB_P_A_S], dt = P[FLYB_P_DT], t_ref = P[FLYB_P_T_REF];
  const float jump = P[FLYB_P_ADAPT_JUMP], a_ad = P[FLYB_P_A_AD], a_std = P[FLYB_P_A_STD];
  const float a_r = P[FLYB_P_A_R], rg = P[FLYB_P_RATE_GAIN], w_syn = P[FLYB_P_W_SYN];
  uint64_t events = 0;
  for (int i = 0; i < n; ++i) {
    const size_t t = (size_t)i * B + b;
    /* per-neuron clocks (brain.py:899-957): the coefficients of this neuron's phase; input that
     * arrives between its updates waits in clock_acc */
    float c_m = a_m, c_s = a_s, c_dt = dt, c_ad = a_ad, c_std = a_std, c_r = a_r, c_rg = rg, c_u = 1.0f,
          c_pois = 1.0f;
    int period = 1, on = 1;
    const float* cf = NULL;
    if (a->clock_k) {
      period = a->clock_k[i];
      on = step % period == 0;
      cf = a->clock_coef + FLYB_CLOCK_NCOEF * (on ? period : 0);
      c_m = cf[FLYB_CLOCK_A_M]; c_s = cf[FLYB_CLOCK_A_S]; c_dt = cf[FLYB_CLOCK_DT]; c_ad = cf[FLYB_CLOCK_A_AD];
      c_std = cf[FLYB_CLOCK_A_STD]; c_r = cf[FLYB_CLOCK_A_R]; c_rg = cf[FLYB_CLOCK_RATE_GAIN]; c_u = cf[FLYB_CLOCK_U];
      c_pois = cf[FLYB_CLOCK_POIS];
    }
    /* 1. synaptic input due now: read and clear the ring slot */
    int64_t due;
    if (a->ring_mode == FLYB_RING_COUNT) {
      int32_t* ring = (int32_t*)a->ring + (size_t)rs * n * B;
      due = ring[t]; ring[t] = 0;
    } else {
      int64_t* ring = (int64_t*)a->ring + (size_t)rs * n * B;
      due = ring[t]; ring[t] = 0;
    }
    if (period > 1) {   /* the reference's per-period accumulator, applied on the update step */
      int64_t* acc = (int64_t*)a->clock_acc + t;
      *acc += due;
      due = on ? *acc : 0;
      if (on) *acc = 0;
    }
    float g = a->g[t];
    g = g * c_s;
    if (due != 0) {
      float inc = a->ring_mode == FLYB_RING_COUNT ? w_syn * (float)due : float_of_fixed(due);
      g = g + inc;
    }
    a->g[t] = g;
    /* the slow tone (brain.py:551-557, 834-837): per class decay plus its delayed input; under
     * clocks the phase's decay and the per-period accumulator of the class (brain.py:905-917) */
    float tone = 0.0f;
    for (int c = 0; c < a->slow_classes; ++c) {
      int64_t* sring = (int64_t*)a->slow_ring[c] + (size_t)rs * n * B;
      int64_t sdue = sring[t]; sring[t] = 0;
      if (period > 1) {
        int64_t* acc = (int64_t*)a->slow_clock_acc[c] + t;
        *acc += sdue;
        sdue = on ? *acc : 0;
        if (on) *acc = 0;
      }
      float sg = a->slow_g[c][t] * (cf ? cf[FLYB_CLOCK_A_SLOW0 + c] : a->slow_decay[c]);
      if (sdue != 0) { float inc = float_of_fixed(sdue); sg = sg + inc; }
      a->slow_g[c][t] = sg;
      tone = tone + sg;
    }
    if (a->slow_classes) a->g_slow[t] = tone;
    /* 2. membrane (brain.py:568-577, 839-843) */
    float th = v_th;
    float target;
    if (a->slow_classes && a->slow_mode == FLYB_SLOW_GAIN) {
      float f = 1.0f + tone / a->slow_norm;
      if (f < a->slow_clip_lo) f = a->slow_clip_lo;
      if (f > a->slow_clip_hi) f = a->slow_clip_hi;
      target = v_rest + g * f;
    } else {
      target = v_rest + g;
    }
    target = target + a->drive[t];
    target = target - a->adapt[t];
    if (a->slow_classes && a->slow_mode == FLYB_SLOW_ADDITIVE) target = target + tone;
    if (a->slow_classes && a->slow_mode == FLYB_SLOW_THRESHOLD) {
      float m = tone < a->slow_th_max ? tone : a->slow_th_max;
      th = -m + v_th;
    }
    float v = a->v[t] - target;
    v = v * c_m;
    v = target + v;
    float ref = a->refrac[t];
    if (ref > 0.0f) v = v_reset;
    ref = ref - c_dt;
    if (ref < 0.0f) ref = 0.0f;
    /* 3. threshold and Poisson forcing (brain.py:845-849) */
    float spike = (v >= th ? 1.0f : 0.0f) * c_u;
    spike = spike * a->active[i];
    if (flags & FLYB_LIF_POISSON) {
      float p = a->poisson_p[t] * c_pois;
      if (p > 0.0f) {
        float u = (flags & FLYB_LIF_EXT_UNIFORM) ? a->uniforms[(size_t)k * n * B + t]
                                                 : oracle_uniform(a->seed, (uint64_t)step, (uint32_t)i, (uint32_t)(a->fly0 + b));
        if (u < p) spike = 1.0f;
      }
    }
    const int fired = spike > 0.0f;
    if (fired) { v = v_reset; ref = t_ref; }
    a->v[t] = v; a->refrac[t] = ref; a->spikes[t] = spike;
    /* 4. adaptation, depression, counters, rate (brain.py:853-868) */
    if (flags & FLYB_LIF_ADAPT) {
      float ad = a->adapt[t] * c_ad;
      ad = ad + spike * (a->adapt_jump ? a->adapt_jump[i] : jump);
      a->adapt[t] = ad;
    }
    float x = spike;
    if (flags & FLYB_LIF_STD) {
      float res = a->res[t];
      x = spike * res;
      if (fired) { float keep = 1.0f - a->std_u[i]; res = res * keep; }
      float dep = 1.0f - res; dep = dep * c_std; res = 1.0f - dep;
      a->res[t] = res;
    }
    if (flags & FLYB_LIF_COUNTS) a->counts[t] = a->counts[t] + spike;
    { float r = a->rate[t] * c_r; r = r + spike * c_rg; a->rate[t] = r; }
    if (fired_out) fired_out[t] = (unsigned char)fired;
    /* 5. deliver D steps later */
    if (x != 0.0f) {
      const int e0 = a->out_ptr[i], e1 = a->out_ptr[i + 1];
      events += (uint64_t)(e1 - e0);
      for (int c = 0; c < a->slow_classes; ++c) {   /* the slow lists carry the same amounts */
        int64_t* sring = (int64_t*)a->slow_ring[c] + (size_t)ws * n * B;
        const int* sp = a->slow_out_ptr[c];
        const int* se = a->slow_out_edge[c];
        for (int e = sp[i]; e < sp[i + 1]; ++e) {
          float w; memcpy(&w, &se[2 * e + 1], sizeof w);
          sring[(size_t)se[2 * e] * B + b] += fixed_of(w, x);
        }
      }
      if (a->ring_mode == FLYB_RING_COUNT) {
        int32_t* ring = (int32_t*)a->ring + (size_t)ws * n * B;
        for (int e = e0; e < e1; ++e) ring[(size_t)a->out_edge[2 * e] * B + b] += a->out_edge[2 * e + 1];
      } else {
        int64_t* ring = (int64_t*)a->ring + (size_t)ws * n * B;
        for (int e = e0; e < e1; ++e) {
          float w; memcpy(&w, &a->out_edge[2 * e + 1], sizeof w);
          ring[(size_t)a->out_edge[2 * e] * B + b] += fixed_of(w, x);
        }
      }
    }
  }
  return events;
}

/* Runs a->nsteps steps on host memory. Same argument struct as the device entry point; the
 * launch fields are ignored. `threads` <= 0 uses every OpenMP thread; flies run in parallel
 * (each fly owns disjoint state and ring columns, so the result does not depend on it). */
int oracle_lif_run(const flyb_lif_args* a, int threads) {
  if (!a || a->n <= 0 || a->batch <= 0 || a->ring_slots <= a->n_delay || a->n_delay < 1) return FLYB_EINVAL;
  const float* P = a->params;
  const size_t W = (size_t)a->n * a->batch, words = (W + 31) / 32;
  unsigned char* fired = a->raster ? (unsigned char*)calloc(W, 1) : NULL;
  if (a->raster && !fired) return FLYB_EINVAL;
  uint64_t total = 0;
  long long step0 = a->step0;
  int ring_pos = a->ring_pos, raster_pos = a->raster_pos;
  if (a->clock) {   /* {step, ring_pos, raster_pos}, advanced below like the device clock */
    step0 = a->clock[0];
    ring_pos = (int)(((a->clock[1] % a->ring_slots) + a->ring_slots) % a->ring_slots);
    raster_pos = a->raster_slots > 0 ? (int)(((a->clock[2] % a->raster_slots) + a->raster_slots) % a->raster_slots) : 0;
  }
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  for (int k = 0; k < a->nsteps; ++k) {
    uint64_t ev = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:ev) if(a->batch > 1)
#endif
    for (int b = 0; b < a->batch; ++b) {
      if ((a->flags & FLYB_LIF_EPISODES) && k >= a->fly_steps[b]) {
        if (fired) for (int i = 0; i < a->n; ++i) fired[(size_t)i * a->batch + b] = 0;
        continue;
      }
      ev += lif_fly_step(a, b, k, P, fired, step0, ring_pos);
    }
    total += ev;
    if (a->raster) {   /* pack the step's spike bits (bit t = i * batch + b) */
      const size_t slot = a->raster_slots > 0 ? (size_t)(((long long)raster_pos + k) % a->raster_slots) : (size_t)k;
      unsigned* row = a->raster + slot * words;
      memset(row, 0, words * sizeof(unsigned));
      for (size_t t = 0; t < W; ++t) if (fired[t]) row[t / 32] |= 1u << (t % 32);
    }
  }
  free(fired);
  if (a->events) a->events[0] += total;
  if (a->clock) {
    a->clock[0] = step0 + a->nsteps;
    a->clock[1] = (ring_pos + a->nsteps) % a->ring_slots;
    a->clock[2] = a->raster_slots > 0 ? (raster_pos + a->nsteps) % a->raster_slots : 0;
  }
  if (a->flags & FLYB_LIF_EPISODES)
    for (int b = 0; b < a->batch; ++b) a->fly_steps[b] = a->fly_steps[b] > a->nsteps ? a->fly_steps[b] - a->nsteps : 0;
  return FLYB_OK;
}

/* ------------------------------------------------------------------ optic substep */
static inline float clip01f(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }
static inline double clip01d(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

/* FP32, the reference order: dr = clip01(v + b) - b; y = W dr (row sum in CSR order);
 * inp = gr*y + pr - ga*adapt; inp = inp + spk; v = inp + (v - inp)*a; adapt = dr + (adapt - dr)*aad.
 * State [m][batch]. Optional histories as in flyb_optic_args. */
int oracle_optic_run(const flyb_optic_args* a, int threads) {
  const int m = a->m, B = a->batch;
  const size_t sz = (size_t)m * B;
  float* dr = (float*)malloc(sz * sizeof(float));
  float* v0 = (float*)malloc(sz * sizeof(float));
  if (!dr || !v0) { free(dr); free(v0); return FLYB_EINVAL; }
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  for (int k = 0; k < a->nsteps; ++k) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long long t = 0; t < (long long)sz; ++t) {
      const float bb = a->b[t / B];
      float r = a->v[t] + bb; r = clip01f(r); dr[t] = r - bb; v0[t] = a->v[t];
    }
    if (a->v_hist) memcpy(a->v_hist + (size_t)k * sz, a->v, sz * sizeof(float));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int i = 0; i < m; ++i) {
      for (int bb = 0; bb < B; ++bb) {
        const size_t t = (size_t)i * B + bb;
        float y = 0.0f;
        for (int e = a->ptr[i]; e < a->ptr[i + 1]; ++e) {
          float w; memcpy(&w, &a->cw[2 * e + 1], sizeof w);
          float p = w * dr[(size_t)a->cw[2 * e] * B + bb]; y = y + p;
        }
        float inp = a->gr * y;
        inp = inp + a->pr[t];
        float ad = a->ga * a->adapt[t];
        inp = inp - ad;
        inp = inp + a->spk[t];
        if (a->inp_hist) a->inp_hist[(size_t)k * sz + t] = inp;
        float dv = v0[t] - inp; dv = dv * a->a[i];
        a->v[t] = inp + dv;
        float old = dr[t];
        float da = a->adapt[t] - old; da = da * a->aad;
        a->adapt[t] = old + da;
      }
    }
  }
  free(dr); free(v0);
  return FLYB_OK;
}

/* FP64 version of the same recurrence on double state (the error reference). */
int oracle_optic_run_f64(int m, int batch, int nsteps, const int* ptr, const int* col, const double* w,
                         double* v, double* adapt, const double* pr, const double* spk,
                         const double* a, const double* b, double gr, double ga, double aad) {
  const size_t sz = (size_t)m * batch;
  double* dr = (double*)malloc(sz * sizeof(double));
  if (!dr) return FLYB_EINVAL;
  for (int k = 0; k < nsteps; ++k) {
    for (size_t t = 0; t < sz; ++t) { double bb = b[t / batch]; dr[t] = clip01d(v[t] + bb) - bb; }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int i = 0; i < m; ++i) {
      for (int bb = 0; bb < batch; ++bb) {
        const size_t t = (size_t)i * batch + bb;
        double y = 0.0;
        for (int e = ptr[i]; e < ptr[i + 1]; ++e) y += w[e] * dr[(size_t)col[e] * batch + bb];
        double inp = gr * y + pr[t] - ga * adapt[t] + spk[t];
        v[t] = inp + (v[t] - inp) * a[i];
        adapt[t] = dr[t] + (adapt[t] - dr[t]) * aad;
      }
    }
  }
  free(dr);
  return FLYB_OK;
}

/* The held-input products with the map / clamp semantics of flyb_spmm (FP32, CSR order). */
int oracle_spmm(const flyb_spmm_args* a) {
  const int B = a->batch;
  for (int i = 0; i < a->rows; ++i) {
    const int yi = a->y_index ? a->y_index[i] : i;
    for (int b = 0; b < B; ++b) {
      float s = 0.0f;
      for (int e = a->ptr[i]; e < a->ptr[i + 1]; ++e) {
        const int j = a->col[e];
        const int xj = a->x_index ? a->x_index[j] : j;
        float x = a->x[(size_t)xj * B + b] / a->x_div;
        x = x < a->x_lo ? a->x_lo : (x > a->x_hi ? a->x_hi : x);
        float p = a->w[e] * x; s = s + p;
      }
      float r = a->alpha * s;
      r = r < a->y_lo ? a->y_lo : (r > a->y_hi ? a->y_hi : r);
      float* y = a->y + (size_t)yi * B + b;
      *y = a->accumulate ? *y + r : r;
    }
  }
  return FLYB_OK;
}
