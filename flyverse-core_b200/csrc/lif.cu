// Event-driven LIF step for sm_100a: fused membrane update, Poisson drive, warp-ballot spike
// compaction and scatter of the spikers' outgoing synapses into an exact delay ring.
//
// Semantics follow flyverse/brain.py:_step_inference (brain.py:829-870) and the fused update of
// flyverse/kernels/neural.cu:18-52; the float spike buffer (brain.py:485-487, 858-865) becomes a
// ring of pending synaptic input. A spike at step t is added to slot (pos(t) + D) mod R, which the
// neuron reads (and clears) D steps later, so the delay equals the reference's D-slot buffer.
//   COUNT ring: int32 signed synapse counts, g += w_syn * sum(count)      (exact integer sum)
//   FIXED ring: int64 Q32.32 mV, each edge adds round(w * x * 2^32)       (exact integer sum)
// Both sums are independent of the order in which red.global.add lands, so rasters and state are
// deterministic and equal to the C restatement in oracle/flyoracle.c bit for bit.
//
// Layout: state [n][batch] (fly-minor), ring [R][n][batch]; work item t = i * batch + b.
#include "common.cuh"

namespace flyb {

struct LifP {
  float v_rest, v_reset, v_th, a_m, a_s, dt, t_ref, jump, a_ad, a_std, a_r, rg, w_syn;
};

struct LifK {
  int n, batch, n_delay, R, flags, nsteps, ring_pos, words, raster_slots, raster_pos, fly0;
  long long step0;
  unsigned long long seed;
  const int* __restrict__ out_ptr;
  const int2* __restrict__ out_edge;
  float* __restrict__ v; float* __restrict__ g; float* __restrict__ refrac; float* __restrict__ adapt;
  float* __restrict__ res; float* __restrict__ rate; float* __restrict__ counts; float* __restrict__ spikes;
  const float* __restrict__ drive; const float* __restrict__ poisson_p;
  const float* __restrict__ active; const float* __restrict__ std_u;
  void* ring;
  const float* __restrict__ uniforms;
  int* fly_steps;
  long long* clock;
  unsigned* raster;
  unsigned long long* events;
  int* status;
  int* sync;
  LifP P;
};

template <int BLOCK>
struct LifSmem {
  int wcnt[BLOCK / 32];
  int woff[BLOCK / 32];
  int total;
  int edges;
  int pre[BLOCK];     // exclusive prefix of spiker out-degrees
  int start[BLOCK];   // first outgoing edge of each spiker
  int fly[BLOCK];     // fly of each spiker
  float x[BLOCK];     // transmitted amount (1, or spike * resource under depression)
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Inclusive warp scan.
__device__ __forceinline__ int warp_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Step counter and ring positions at the start of a launch: from the device clock when one is
// given (CUDA-graph replays then advance them), else from the host arguments.
struct Clk {
  long long step0;
  int ring_pos, raster_pos;
};

__device__ __forceinline__ Clk read_clock(const LifK& k) {
  if (!k.clock) return Clk{k.step0, k.ring_pos, k.raster_pos};
  const long long r = k.clock[1], h = k.clock[2];
  return Clk{k.clock[0], (int)(((r % k.R) + k.R) % k.R), k.raster_slots > 0 ? (int)(((h % k.raster_slots) + k.raster_slots) % k.raster_slots) : 0};
}

// After the last step: advance the device clock and lower the per-fly remaining-step counters.
__device__ __forceinline__ void advance_clock(const LifK& k, const Clk& c) {
  if (threadIdx.x == 0 && k.clock) {
    k.clock[0] = c.step0 + k.nsteps;
    k.clock[1] = (c.ring_pos + k.nsteps) % k.R;
    k.clock[2] = k.raster_slots > 0 ? (c.raster_pos + k.nsteps) % k.raster_slots : 0;
  }
  if (k.flags & FLYB_LIF_EPISODES)
    for (int b = threadIdx.x; b < k.batch; b += blockDim.x) k.fly_steps[b] = max(k.fly_steps[b] - k.nsteps, 0);
}

// One block processes work items [base, base + BLOCK) of local step `s`: update, then deliver.
template <int BLOCK, bool FIXED>
__device__ __forceinline__ void lif_chunk(const LifK& k, const Clk& clk, int s, long long base, LifSmem<BLOCK>& sm) {
  const long long W = (long long)k.n * k.batch;
  const long long t = base + threadIdx.x;
  const int rs = (int)(((long long)clk.ring_pos + s) % k.R);
  const int ws = (int)(((long long)clk.ring_pos + s + k.n_delay) % k.R);
  const size_t slot = (size_t)W;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const LifP& P = k.P;
  bool fired = false;
  float x = 0.0f;
  int i = 0, b = 0;
  if (t < W) {
    i = (int)(t / k.batch);
    b = (int)(t - (long long)i * k.batch);
    const bool live = !(k.flags & FLYB_LIF_EPISODES) || s < k.fly_steps[b];
    if (live) {
      // 1. input due now from the ring (read; clear only what was non-zero)
      long long c;
      if (FIXED) {
        long long* r = (long long*)k.ring + (size_t)rs * slot + t;
        c = *r;
        if (c) *r = 0;
      } else {
        int* r = (int*)k.ring + (size_t)rs * slot + t;
        c = *r;
        if (c) *r = 0;
      }
      const float act = k.active[i];
      const float p = (k.flags & FLYB_LIF_POISSON) ? k.poisson_p[t] : 0.0f;
      float vv = k.v[t], gg = k.g[t], ref = k.refrac[t];
      const float ad0 = k.adapt[t], dv = k.drive[t];
      bool skip = false;
      if ((k.flags & FLYB_LIF_SKIP_FROZEN) && act == 0.0f && p == 0.0f && c == 0) {
        // frozen cell at rest: the update would leave it unchanged (neural.cu:24-26)
        skip = vv == P.v_rest && gg == 0.0f && dv == 0.0f && ad0 == 0.0f && ref == 0.0f &&
               k.rate[t] == 0.0f && k.spikes[t] == 0.0f && k.res[t] == 1.0f;
      }
      if (!skip) {
        gg = gg * P.a_s;
        if (c) {
          const float inc = FIXED ? __double2float_rn((double)c * (1.0 / 4294967296.0)) : P.w_syn * (float)c;
          gg = gg + inc;
        }
        k.g[t] = gg;
        // 2. membrane, exponential Euler with g and drive held (brain.py:839-843)
        float target = P.v_rest + gg;
        target = target + dv;
        target = target - ad0;
        float u = vv - target;
        u = u * P.a_m;
        vv = target + u;
        if (ref > 0.0f) vv = P.v_reset;
        ref = ref - P.dt;
        if (ref < 0.0f) ref = 0.0f;
        // 3. threshold x active, Poisson forcing (brain.py:845-849)
        float spike = (vv >= P.v_th ? 1.0f : 0.0f) * act;
        if (p > 0.0f) {
          const float un = (k.flags & FLYB_LIF_EXT_UNIFORM)
                               ? k.uniforms[(size_t)s * slot + t]
                               : philox_uniform(k.seed, clk.step0 + s, (uint32_t)i, (uint32_t)(k.fly0 + b));
          if (un < p) spike = 1.0f;
        }
        fired = spike > 0.0f;
        if (fired) { vv = P.v_reset; ref = P.t_ref; }
        k.v[t] = vv;
        k.refrac[t] = ref;
        k.spikes[t] = spike;
        // 4. adaptation, depression, counters, rate (brain.py:853-868)
        if (k.flags & FLYB_LIF_ADAPT) { float ad = ad0 * P.a_ad; ad = ad + spike * P.jump; k.adapt[t] = ad; }
        x = spike;
        if (k.flags & FLYB_LIF_STD) {
          float rr = k.res[t];
          x = spike * rr;
          if (fired) { const float keep = 1.0f - k.std_u[i]; rr = rr * keep; }
          float dep = 1.0f - rr;
          dep = dep * P.a_std;
          rr = 1.0f - dep;
          k.res[t] = rr;
        }
        if (k.flags & FLYB_LIF_COUNTS) k.counts[t] = k.counts[t] + spike;
        float rt = k.rate[t] * P.a_r;
        rt = rt + spike * P.rg;
        k.rate[t] = rt;
      }
    }
  }
  // raster word of this warp (flat bit order t)
  const unsigned fb = __ballot_sync(0xffffffffu, fired);
  if (k.raster && lane == 0 && base + warp * 32 < W) {
    const size_t slot = k.raster_slots > 0 ? (size_t)(((long long)clk.raster_pos + s) % k.raster_slots) : (size_t)s;
    k.raster[slot * k.words + (size_t)((base >> 5) + warp)] = fb;
  }
  // 5. compact the transmitting cells of this block (warp ballot + block prefix)
  const unsigned tb = __ballot_sync(0xffffffffu, x != 0.0f);
  if (lane == 0) sm.wcnt[warp] = __popc(tb);
  __syncthreads();
  if (warp == 0) {
    const int c = lane < BLOCK / 32 ? sm.wcnt[lane] : 0;
    const int inc = warp_scan(c);
    if (lane < BLOCK / 32) sm.woff[lane] = inc - c;
    if (lane == 31) sm.total = inc;
  }
  __syncthreads();
  const int L = sm.total;
  if (L == 0) return;   // block-uniform
  int deg = 0;
  if (x != 0.0f) {
    const int pos = sm.woff[warp] + __popc(tb & lanemask_lt());
    const int e0 = k.out_ptr[i];
    deg = k.out_ptr[i + 1] - e0;
    sm.start[pos] = e0;
    sm.fly[pos] = b;
    sm.x[pos] = x;
    sm.pre[pos] = deg;   // degree for now; turned into an exclusive prefix below
  }
  __syncthreads();
  // exclusive prefix of degrees over the L spikers
  {
    const int d = threadIdx.x < L ? sm.pre[threadIdx.x] : 0;
    const int inc = warp_scan(d);
    if (lane == 31) sm.wcnt[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const int c = lane < BLOCK / 32 ? sm.wcnt[lane] : 0;
      const int winc = warp_scan(c);
      if (lane < BLOCK / 32) sm.woff[lane] = winc - c;
      if (lane == 31) sm.edges = winc;
    }
    __syncthreads();
    if (threadIdx.x < L) sm.pre[threadIdx.x] = sm.woff[warp] + inc - d;
    __syncthreads();
  }
  const int E = sm.edges;
  // 6. block-wide, edge-parallel delivery into slot ws: thread q takes edges q, q+BLOCK, ...
  for (int q = threadIdx.x; q < E; q += BLOCK) {
    int lo = 0, hi = L - 1;   // last spiker with pre <= q
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sm.pre[mid] <= q) lo = mid; else hi = mid - 1;
    }
    const int2 ed = __ldg(&k.out_edge[sm.start[lo] + (q - sm.pre[lo])]);
    const size_t dst = (size_t)ws * slot + (size_t)ed.x * k.batch + sm.fly[lo];
    if (FIXED) {
      const long long f = __double2ll_rn((double)__int_as_float(ed.y) * (double)sm.x[lo] * 4294967296.0);
      atomicAdd((unsigned long long*)k.ring + dst, (unsigned long long)f);
    } else {
      atomicAdd((int*)k.ring + dst, ed.y);
    }
  }
  if (k.events && threadIdx.x == 0) atomicAdd(k.events, (unsigned long long)E);
  __syncthreads();   // shared lists are reused by the next chunk
}

template <int BLOCK, bool FIXED>
__global__ void __launch_bounds__(BLOCK) lif_step_kernel(LifK k, int s) {
  __shared__ LifSmem<BLOCK> sm;
  const Clk clk = read_clock(k);
  lif_chunk<BLOCK, FIXED>(k, clk, s, (long long)blockIdx.x * BLOCK, sm);
}

__global__ void lif_advance_kernel(LifK k) { advance_clock(k, read_clock(k)); }

template <int BLOCK, bool FIXED>
__global__ void __launch_bounds__(BLOCK) lif_persistent_kernel(LifK k) {
  __shared__ LifSmem<BLOCK> sm;
  const long long W = (long long)k.n * k.batch;
  const Clk clk = read_clock(k);
  int generation = 0;
  for (int s = 0; s < k.nsteps; ++s) {
    for (long long base = (long long)blockIdx.x * BLOCK; base < W; base += (long long)gridDim.x * BLOCK)
      lif_chunk<BLOCK, FIXED>(k, clk, s, base, sm);
    // the next step writes the slot this step read: every block must be done with it
    if (!grid_barrier(k.sync, k.status, generation, s)) return;
  }
  // every block has read the clock and the episode counters: advance them
  if (blockIdx.x == 0) advance_clock(k, clk);
}

template <int BLOCK, bool FIXED>
static void* persistent_fn() { return (void*)lif_persistent_kernel<BLOCK, FIXED>; }

template <int BLOCK, bool FIXED>
static int run_lif(const LifK& k, int launch, int grid_cap, cudaStream_t st) {
  const long long W = (long long)k.n * k.batch;
  const long long chunks = (W + BLOCK - 1) / BLOCK;
  if (launch == FLYB_LAUNCH_STEP) {
    for (int s = 0; s < k.nsteps; ++s) {
      lif_step_kernel<BLOCK, FIXED><<<(unsigned)chunks, BLOCK, 0, st>>>(k, s);
      FLYB_CHECK_LAUNCH();
    }
    if (k.clock || (k.flags & FLYB_LIF_EPISODES)) {
      lif_advance_kernel<<<1, 256, 0, st>>>(k);
      FLYB_CHECK_LAUNCH();
    }
    return 0;
  }
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lif_persistent_kernel<BLOCK, FIXED>, BLOCK, 0);
  long long grid = (long long)sms * per_sm;
  if (grid > chunks) grid = chunks;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  if (grid < 1) return FLYB_ECOOP;
  cudaError_t e = cudaMemsetAsync(k.sync, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  LifK kk = k;
  void* args[] = {&kk};
  e = cudaLaunchCooperativeKernel(persistent_fn<BLOCK, FIXED>(), dim3((unsigned)grid), dim3(BLOCK), args, 0, st);
  return (int)e;
}

// ------------------------------------------------------------------ ring deposit (checkpoint import)
template <bool FIXED>
__global__ void ring_deposit_kernel(int n, int batch, const int* __restrict__ out_ptr, const int2* __restrict__ out_edge,
                                    const float* __restrict__ x, void* ring) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * batch) return;
  const float xv = x[t];
  if (xv == 0.0f) return;
  const int i = (int)(t / batch), b = (int)(t - (long long)i * batch);
  for (int e = out_ptr[i]; e < out_ptr[i + 1]; ++e) {
    const int2 ed = out_edge[e];
    const size_t dst = (size_t)ed.x * batch + b;
    if (FIXED) {
      const long long f = __double2ll_rn((double)__int_as_float(ed.y) * (double)xv * 4294967296.0);
      atomicAdd((unsigned long long*)ring + dst, (unsigned long long)f);
    } else {
      atomicAdd((int*)ring + dst, ed.y);
    }
  }
}

// ------------------------------------------------------------------ reference-compatible launchers
// Batch-major (B, N) state, float spike buffer; same flags and pointer order as neural.cu:11-60.
struct RefLif {
  float *v, *g, *drive, *adapt, *refrac, *active, *prob, *rnd;
  float *res, *std_u, *spikes, *out, *rate, *counts, *p, *phase;
};

__global__ void ref_lif_kernel(RefLif s, int n, long long total, int flags) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int i = (int)(t % n);
  if ((flags & 32) && s.active[i] == 0 && (!(flags & 1) || s.prob[t] == 0) && s.v[t] == s.p[0] && s.g[t] == 0 &&
      s.drive[t] == 0 && s.adapt[t] == 0 && s.refrac[t] == 0 && s.rate[t] == 0 && s.spikes[t] == 0 && s.out[t] == 0 &&
      s.res[t] == 1)
    return;
  float am = s.p[3], dt = s.p[4], aad = s.p[7], ast = s.p[8], ar = s.p[9], rg = s.p[10], u = 1.0f, pois = 1.0f;
  if (flags & 16) {
    am = s.phase[i]; dt = s.phase[n + i]; aad = s.phase[2 * n + i]; ast = s.phase[3 * n + i];
    ar = s.phase[4 * n + i]; rg = s.phase[5 * n + i]; u = s.phase[6 * n + i]; pois = s.phase[7 * n + i];
  }
  float target = s.p[0] + s.g[t];
  target = target + s.drive[t];
  target = target - s.adapt[t];
  float v = s.v[t] - target;
  v = v * am;
  v = target + v;
  float ref = s.refrac[t];
  if (ref > 0.0f) v = s.p[1];
  ref = ref - dt;
  if (ref < 0.0f) ref = 0.0f;
  float spike = (v >= s.p[2] ? 1.0f : 0.0f) * u;
  spike = spike * s.active[i];
  if (flags & 1) { const float q = s.prob[t] * pois; if (s.rnd[t] < q) spike = fmaxf(spike, 1.0f); }
  const bool fired = spike > 0.0f;
  if (fired) { v = s.p[1]; ref = s.p[5]; }
  s.v[t] = v; s.refrac[t] = ref; s.spikes[t] = spike;
  if (flags & 8) s.adapt[t] = fmaf(spike, s.p[6], s.adapt[t] * aad);
  if (flags & 2) {
    float resource = s.res[t];
    s.out[t] = spike * resource;
    if (fired) { const float keep = 1.0f - s.std_u[i]; resource = resource * keep; }
    float dep = 1.0f - resource;
    dep = dep * ast;
    s.res[t] = 1.0f - dep;
  } else {
    s.out[t] = spike;
  }
  if (flags & 4) s.counts[t] = s.counts[t] + spike;
  float r = s.rate[t] * ar;
  r = r + spike * rg;
  s.rate[t] = r;
}

// One warp per (fly, presynaptic column); silent columns exit before touching edges.
template <typename W>
__global__ void ref_events_kernel(const int* __restrict__ ptr, const int* __restrict__ idx, const W* __restrict__ w,
                                  const float* __restrict__ x, float* g, const int* __restrict__ pre_ids, int n,
                                  int batch, int count) {
  const int lane = threadIdx.x & 31;
  const long long gid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int size = count < 0 ? n : count;
  if (gid >= (long long)size * batch) return;
  const int b = (int)(gid / size);
  const int k = (int)(gid - (long long)b * size);
  const int pre = count < 0 ? k : pre_ids[k];
  const float value = x[(size_t)b * n + pre];
  if (value == 0.0f) return;
  for (int e = ptr[pre] + lane; e < ptr[pre + 1]; e += 32) {
    const float p = (float)w[e] * value;
    atomicAdd(g + (size_t)b * n + idx[e], p);
  }
}

int lif_blocks_per_sm(int block) {
  int b = 0;
  if (block == 128) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<128, false>, 128, 0);
  else if (block == 512) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<512, false>, 512, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<256, false>, 256, 0);
  return b;
}

}  // namespace flyb

using namespace flyb;

FLYB_API int flyb_lif_run(const flyb_lif_args* a, void* stream) {
  if (!a || a->n <= 0 || a->batch <= 0 || a->n_delay < 1 || a->ring_slots < a->n_delay + 1 || a->nsteps < 0 ||
      !a->out_ptr || !a->v || !a->g || !a->refrac || !a->adapt || !a->res || !a->rate ||
      !a->counts || !a->spikes || !a->drive || !a->poisson_p || !a->active || !a->params || !a->ring ||
      (a->ring_mode != FLYB_RING_COUNT && a->ring_mode != FLYB_RING_FIXED))
    return FLYB_EINVAL;
  if ((long long)a->n * a->batch >= (1ll << 31)) return FLYB_ETOOBIG;
  if ((a->flags & FLYB_LIF_STD) && (!a->std_u || a->ring_mode != FLYB_RING_FIXED)) return FLYB_EINVAL;
  if ((a->flags & FLYB_LIF_EXT_UNIFORM) && !a->uniforms) return FLYB_EINVAL;
  if ((a->flags & FLYB_LIF_EPISODES) && !a->fly_steps) return FLYB_EINVAL;
  if (a->launch == FLYB_LAUNCH_PERSISTENT && (!a->sync || !a->status)) return FLYB_EINVAL;
  if (a->nsteps == 0) return 0;
  LifK k;
  k.n = a->n; k.batch = a->batch; k.n_delay = a->n_delay; k.R = a->ring_slots; k.flags = a->flags;
  k.nsteps = a->nsteps; k.ring_pos = ((a->ring_pos % k.R) + k.R) % k.R;
  k.words = (int)(((long long)a->n * a->batch + 31) / 32);
  k.step0 = a->step0; k.seed = a->seed;
  k.out_ptr = a->out_ptr; k.out_edge = (const int2*)a->out_edge;
  k.v = a->v; k.g = a->g; k.refrac = a->refrac; k.adapt = a->adapt; k.res = a->res; k.rate = a->rate;
  k.counts = a->counts; k.spikes = a->spikes; k.drive = a->drive; k.poisson_p = a->poisson_p;
  k.active = a->active; k.std_u = a->std_u; k.ring = a->ring; k.uniforms = a->uniforms; k.fly_steps = a->fly_steps;
  k.clock = a->clock;
  k.raster = a->raster; k.raster_slots = a->raster_slots; k.raster_pos = a->raster_pos; k.fly0 = a->fly0;
  k.events = a->events; k.status = a->status; k.sync = a->sync;
  const float* P = a->params;
  k.P = LifP{P[FLYB_P_V_REST], P[FLYB_P_V_RESET], P[FLYB_P_V_TH], P[FLYB_P_A_M], P[FLYB_P_A_S], P[FLYB_P_DT],
             P[FLYB_P_T_REF], P[FLYB_P_ADAPT_JUMP], P[FLYB_P_A_AD], P[FLYB_P_A_STD], P[FLYB_P_A_R],
             P[FLYB_P_RATE_GAIN], P[FLYB_P_W_SYN]};
  cudaStream_t st = (cudaStream_t)stream;
  const bool fixed = a->ring_mode == FLYB_RING_FIXED;
  const int block = a->block ? a->block : 256;
  switch (block) {
    case 128: return fixed ? run_lif<128, true>(k, a->launch, a->grid, st) : run_lif<128, false>(k, a->launch, a->grid, st);
    case 256: return fixed ? run_lif<256, true>(k, a->launch, a->grid, st) : run_lif<256, false>(k, a->launch, a->grid, st);
    case 512: return fixed ? run_lif<512, true>(k, a->launch, a->grid, st) : run_lif<512, false>(k, a->launch, a->grid, st);
    default: return FLYB_EINVAL;
  }
}

FLYB_API int flyb_ring_deposit(int n, int batch, int ring_mode, const int* out_ptr, const int* out_edge,
                               const float* x, void* ring_slot, void* stream) {
  if (n <= 0 || batch <= 0 || !out_ptr || !out_edge || !x || !ring_slot) return FLYB_EINVAL;
  const long long W = (long long)n * batch;
  const unsigned blocks = (unsigned)((W + 255) / 256);
  if (ring_mode == FLYB_RING_FIXED)
    ring_deposit_kernel<true><<<blocks, 256, 0, (cudaStream_t)stream>>>(n, batch, out_ptr, (const int2*)out_edge, x, ring_slot);
  else if (ring_mode == FLYB_RING_COUNT)
    ring_deposit_kernel<false><<<blocks, 256, 0, (cudaStream_t)stream>>>(n, batch, out_ptr, (const int2*)out_edge, x, ring_slot);
  else
    return FLYB_EINVAL;
  return (int)cudaGetLastError();
}

FLYB_API int launch_lif(void** p, int n, int batch, int flags, void* stream) {
  RefLif s{(float*)p[0], (float*)p[1], (float*)p[2], (float*)p[3], (float*)p[4], (float*)p[5], (float*)p[6], (float*)p[7],
           (float*)p[8], (float*)p[9], (float*)p[10], (float*)p[11], (float*)p[12], (float*)p[13], (float*)p[14], (float*)p[15]};
  const long long total = (long long)n * batch;
  if (total > 0) ref_lif_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(s, n, total, flags);
  return (int)cudaGetLastError();
}

FLYB_API int launch_events(void** p, int n, int batch, int half, int count, void* stream) {
  const long long warps = (long long)(count < 0 ? n : count) * batch;
  const unsigned blocks = (unsigned)((warps + 7) / 8);
  if (blocks) {
    if (half)
      ref_events_kernel<__half><<<blocks, 256, 0, (cudaStream_t)stream>>>((int*)p[0], (int*)p[1], (__half*)p[2], (float*)p[3],
                                                                          (float*)p[4], (int*)p[5], n, batch, count);
    else
      ref_events_kernel<float><<<blocks, 256, 0, (cudaStream_t)stream>>>((int*)p[0], (int*)p[1], (float*)p[2], (float*)p[3],
                                                                         (float*)p[4], (int*)p[5], n, batch, count);
  }
  return (int)cudaGetLastError();
}
