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
#include <type_traits>

#include "common.cuh"

namespace flyb {

struct LifP {
  float v_rest, v_reset, v_th, a_m, a_s, dt, t_ref, jump, a_ad, a_std, a_r, rg, w_syn;
};

struct LifK {
  int n, batch, n_delay, R, flags, nsteps, ring_pos, words, raster_slots, raster_pos, fly0;
  unsigned bdiv_m;      // item t -> neuron t / batch as (umulhi(t, bdiv_m) + t) >> bdiv_s (t < 2^31)
  int bdiv_s;
  int t_begin, t_end;   // items [t_begin, t_end) = neurons [n_first, n_first + n_count) x batch
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
  int4* spike_list;   // deferred delivery: {fly, first edge, edges, x bits} per chunk of a spiker's edges
  unsigned* spike_n;  // entries appended this step
  long long spike_cap;
  const float* __restrict__ adapt_jump;   // per-neuron adaptation jump, or null (P.jump)
  const unsigned char* __restrict__ clock_k;  // per-neuron update period, or null (every step)
  const float* __restrict__ clock_coef;       // [max period + 1][FLYB_CLOCK_NCOEF]
  long long* clock_acc;                       // [n][batch] input pending until the next update
  long long* slow_clock_acc[FLYB_SLOW_MAX_CLASSES];  // the same per slow class (clocks + tone)
  int slow_classes, slow_mode;                // slow receptor tone (0 classes: none)
  float slow_norm, slow_clip_lo, slow_clip_hi, slow_th_max;
  float slow_decay[FLYB_SLOW_MAX_CLASSES];
  const int* slow_out_ptr[FLYB_SLOW_MAX_CLASSES];
  const int2* slow_out_edge[FLYB_SLOW_MAX_CLASSES];
  long long* slow_ring[FLYB_SLOW_MAX_CLASSES];
  float* slow_g[FLYB_SLOW_MAX_CLASSES];
  float* g_slow;
  const int* __restrict__ pull_ptr;            // pull delivery: first 32-entry input chunk per row
  const int* __restrict__ pull_pre;            // [chunks][32] presynaptic neuron (-1: padding), or
                                               // packed: neuron | excess << 24 (0xFFFFFF: padding)
  const unsigned* __restrict__ pull_planes;    // [chunks][pull_nplanes] count bit planes
  int pull_nplanes;                            // plane stride per chunk (16), or 0: packed entries
  const int* __restrict__ pull_meta;           // per chunk: base count << 5 | planes used
  int pull_group;                              // L: steps a pull delivers together
  int pull_phase;                              // runs that pull themselves: first step's index mod L
  unsigned* pull_bits;                         // [2][words][L] spike words of the last two groups
  long long* pull_state;                       // {first undelivered step, its ring position, counter}
  int pull_grid;                               // blocks of a pull launch (0: one wave)
  int pull_group_log2;                         // log2(pull_group)
  LifP P;
};

// Out-edges per deferred-delivery entry: a spiker's edge list is cut into chunks of at most this
// many, so one block of the scatter kernel never walks more (out-degrees reach 10^4 and beyond).
constexpr int kEdgeChunk = 1024;

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

// Division by the batch width with a precomputed multiplier (Granlund & Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994: the round-up variant with an added dividend):
// exact for every 0 <= t < 2^31.
__device__ __forceinline__ int neuron_of(const LifK& k, int t) {
  return (int)((__umulhi((unsigned)t, k.bdiv_m) + (unsigned)t) >> k.bdiv_s);
}

static void batch_divider(int d, unsigned* m, int* s) {
  int l = 0;
  while ((1ll << l) < d) ++l;
  *m = (unsigned)(((1ull << 32) * ((1ull << l) - (unsigned long long)d)) / (unsigned long long)d + 1ull);
  *s = l;
}

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

// v mod m in [0, m) for m > 0: a compare when v already is in range (the clock keeps its positions
// reduced), a 64-bit modulo only otherwise. Every thread reads the clock, so this stays cheap.
__device__ __forceinline__ int wrap_pos(long long v, int m) {
  if (v >= 0 && v < m) return (int)v;
  const long long q = v % m;
  return (int)(q < 0 ? q + m : q);
}

// (pos + d) mod m for 0 <= pos < m and d >= 0, in 32-bit arithmetic.
__device__ __forceinline__ int slot_after(int pos, int d, int m) {
  const int v = pos + d;
  return v < m ? v : v % m;
}

__device__ __forceinline__ Clk read_clock(const LifK& k) {
  if (!k.clock) return Clk{k.step0, k.ring_pos, k.raster_pos};
  return Clk{k.clock[0], wrap_pos(k.clock[1], k.R), k.raster_slots > 0 ? wrap_pos(k.clock[2], k.raster_slots) : 0};
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

// Vector access of IPT consecutive items (16-byte loads / stores when IPT == 4).
template <int IPT, typename T>
__device__ __forceinline__ void vload(const T* p, T (&x)[IPT]) {
  if constexpr (IPT == 2 && sizeof(T) == 4) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    x[0] = *reinterpret_cast<const T*>(&q.x); x[1] = *reinterpret_cast<const T*>(&q.y);
  } else if constexpr (IPT == 2 && sizeof(T) == 8) {
    const longlong2 a = *reinterpret_cast<const longlong2*>(p);
    x[0] = *reinterpret_cast<const T*>(&a.x); x[1] = *reinterpret_cast<const T*>(&a.y);
  } else if constexpr (IPT == 4 && sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    x[0] = *reinterpret_cast<const T*>(&q.x);
    x[1] = *reinterpret_cast<const T*>(&q.y); x[2] = *reinterpret_cast<const T*>(&q.z); x[3] = *reinterpret_cast<const T*>(&q.w);
  } else if constexpr (IPT == 4 && sizeof(T) == 8) {
    const longlong2 a = *reinterpret_cast<const longlong2*>(p), b = *reinterpret_cast<const longlong2*>(p + 2);
    x[0] = *reinterpret_cast<const T*>(&a.x); x[1] = *reinterpret_cast<const T*>(&a.y);
    x[2] = *reinterpret_cast<const T*>(&b.x); x[3] = *reinterpret_cast<const T*>(&b.y);
  } else {
#pragma unroll
    for (int q = 0; q < IPT; ++q) x[q] = p[q];
  }
}

template <int IPT, typename T>
__device__ __forceinline__ void vstore(T* p, const T (&x)[IPT]) {
  if constexpr (IPT == 2 && sizeof(T) == 4) {
    float2 q;
    q.x = *reinterpret_cast<const float*>(&x[0]); q.y = *reinterpret_cast<const float*>(&x[1]);
    *reinterpret_cast<float2*>(p) = q;
  } else if constexpr (IPT == 2 && sizeof(T) == 8) {
    longlong2 a;
    a.x = *reinterpret_cast<const long long*>(&x[0]); a.y = *reinterpret_cast<const long long*>(&x[1]);
    *reinterpret_cast<longlong2*>(p) = a;
  } else if constexpr (IPT == 4 && sizeof(T) == 4) {
    float4 q;
    q.x = *reinterpret_cast<const float*>(&x[0]); q.y = *reinterpret_cast<const float*>(&x[1]);
    q.z = *reinterpret_cast<const float*>(&x[2]); q.w = *reinterpret_cast<const float*>(&x[3]);
    *reinterpret_cast<float4*>(p) = q;
  } else if constexpr (IPT == 4 && sizeof(T) == 8) {
    longlong2 a, b;
    a.x = *reinterpret_cast<const long long*>(&x[0]); a.y = *reinterpret_cast<const long long*>(&x[1]);
    b.x = *reinterpret_cast<const long long*>(&x[2]); b.y = *reinterpret_cast<const long long*>(&x[3]);
    *reinterpret_cast<longlong2*>(p) = a;
    *reinterpret_cast<longlong2*>(p + 2) = b;
  } else {
#pragma unroll
    for (int q = 0; q < IPT; ++q) p[q] = x[q];
  }
}

// Steps 1-4 of one live item (neuron i, fly b) whose ring entry due now is c, in the reference
// order (brain.py:829-868, neural.cu:18-52), every float operation separately rounded. Returns the
// spike value; x is the amount transmitted (the spike, times the resource under depression).
template <bool FIXED, typename RingT>
__device__ __forceinline__ float lif_update(const LifK& k, const Clk& clk, int s, size_t slot, size_t t, int i, int b,
                                            RingT c, float act, float pp, float dv, float& v, float& g, float& ref,
                                            float& ad, float& rt, float& cn, float& rr, float& x) {
  const LifP& P = k.P;
  const int flags = k.flags;
  // 1. synaptic input due now
  float g1 = g * P.a_s;
  if (c) {
    const float inc = FIXED ? __double2float_rn((double)c * (1.0 / 4294967296.0)) : P.w_syn * (float)c;
    g1 = g1 + inc;
  }
  g = g1;
  // 2. membrane, exponential Euler with g and drive held (brain.py:839-843)
  float target = P.v_rest + g1;
  target = target + dv;
  target = target - ad;
  float u = v - target;
  u = u * P.a_m;
  float v1 = target + u;
  float r1 = ref;
  if (r1 > 0.0f) v1 = P.v_reset;
  r1 = r1 - P.dt;
  if (r1 < 0.0f) r1 = 0.0f;
  // 3. threshold x active, Poisson forcing (brain.py:845-849)
  float spike = (v1 >= P.v_th ? 1.0f : 0.0f) * act;
  if (pp > 0.0f) {
    const float un = (flags & FLYB_LIF_EXT_UNIFORM)
                         ? k.uniforms[(size_t)s * slot + t]
                         : philox_uniform(k.seed, clk.step0 + s, (uint32_t)i, (uint32_t)(k.fly0 + b));
    if (un < pp) spike = 1.0f;
  }
  const bool fired = spike > 0.0f;
  if (fired) { v1 = P.v_reset; r1 = P.t_ref; }
  v = v1;
  ref = r1;
  // 4. adaptation, depression, counters, rate (brain.py:853-868)
  if (flags & FLYB_LIF_ADAPT) {
    float a1 = ad * P.a_ad;
    a1 = a1 + spike * (k.adapt_jump ? __ldg(&k.adapt_jump[i]) : P.jump);
    ad = a1;
  }
  x = spike;
  if (flags & FLYB_LIF_STD) {
    float r2 = rr;
    x = spike * r2;
    if (fired) { const float keep = 1.0f - k.std_u[i]; r2 = r2 * keep; }
    float dep = 1.0f - r2;
    dep = dep * P.a_std;
    rr = 1.0f - dep;
  }
  if (flags & FLYB_LIF_COUNTS) cn = cn + spike;
  float r3 = rt * P.a_r;
  r3 = r3 + spike * P.rg;
  rt = r3;
  return spike;
}

// 5-6. Compact the transmitting items of a block (per-thread bits over IPT items, warp scan, block
// prefix), prefix their out-degrees, then deliver every out-edge edge-parallel into ring slot `ws`
// with integer red.global.add. tx bit q of a thread describes its item q: neuron iq[q], fly bq[q],
// transmitted amount xq[q].
template <int BLOCK, bool FIXED, int IPT>
__device__ __forceinline__ void deliver(const LifK& k, LifSmem<BLOCK * IPT>& sm, unsigned tx_bits, const int (&iq)[IPT],
                                        const int (&bq)[IPT], const float (&xq)[IPT], int ws, size_t slot) {
  constexpr int NW = BLOCK / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cnt = __popc(tx_bits);
  const int incl = warp_scan(cnt);
  if (lane == 31) sm.wcnt[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int c = lane < NW ? sm.wcnt[lane] : 0;
    const int inc = warp_scan(c);
    if (lane < NW) sm.woff[lane] = inc - c;
    if (lane == 31) sm.total = inc;
  }
  __syncthreads();
  const int L = sm.total;
  if (L == 0) return;   // block-uniform
  {
    int pos = sm.woff[warp] + incl - cnt;
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      if (tx_bits & (1u << q)) {
        const int e0 = k.out_ptr[iq[q]];
        sm.start[pos] = e0;
        sm.fly[pos] = bq[q];
        sm.x[pos] = xq[q];
        sm.pre[pos] = k.out_ptr[iq[q] + 1] - e0;   // degree for now; exclusive prefix below
        ++pos;
      }
    }
  }
  __syncthreads();
  // exclusive prefix of the degrees over the L transmitting items (thread j: entries j*IPT..)
  {
    int d[IPT], sum = 0;
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const int e = threadIdx.x * IPT + q;
      d[q] = e < L ? sm.pre[e] : 0;
      sum += d[q];
    }
    const int inc = warp_scan(sum);
    if (lane == 31) sm.wcnt[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const int c = lane < NW ? sm.wcnt[lane] : 0;
      const int winc = warp_scan(c);
      if (lane < NW) sm.woff[lane] = winc - c;
      if (lane == 31) sm.edges = winc;
    }
    __syncthreads();
    int run = sm.woff[warp] + inc - sum;
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const int e = threadIdx.x * IPT + q;
      if (e < L) sm.pre[e] = run;
      run += d[q];
    }
    __syncthreads();
  }
  const int E = sm.edges;
  // 6. block-wide, edge-parallel delivery into slot ws: thread j takes edges j, j+BLOCK, ...
  for (int q = threadIdx.x; q < E; q += BLOCK) {
    int lo = 0, hi = L - 1;   // last transmitting item with pre <= q
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

// Deferred delivery, update side: a warp with transmitting items reserves list entries with one
// atomicAdd (each item takes one entry per kEdgeChunk of its out-edges) and writes them; the
// scatter kernel of the same step delivers them. Entries beyond spike_cap are not written and set
// FLYB_ETOOBIG (the host sizes the list so that this cannot happen).
template <int IPT>
__device__ __forceinline__ void append_spikes(const LifK& k, int s, unsigned tx_bits, const int (&iq)[IPT],
                                              const int (&bq)[IPT], const float (&xq)[IPT]) {
  const int lane = threadIdx.x & 31;
  if (!__any_sync(0xffffffffu, tx_bits != 0)) return;   // nearly every warp: nothing fired
  int e0[IPT], deg[IPT], cnt = 0;
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    e0[q] = 0; deg[q] = 0;
    if (tx_bits & (1u << q)) {
      e0[q] = k.out_ptr[iq[q]];
      deg[q] = k.out_ptr[iq[q] + 1] - e0[q];
      cnt += (deg[q] + kEdgeChunk - 1) / kEdgeChunk;
    }
  }
  const int incl = warp_scan(cnt);
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned base = 0;
  if (lane == 31 && total) base = atomicAdd(k.spike_n, (unsigned)total);
  base = __shfl_sync(0xffffffffu, base, 31);
  long long pos = (long long)base + incl - cnt;
#pragma unroll
  for (int q = 0; q < IPT; ++q) {
    for (int c = 0; c < deg[q]; c += kEdgeChunk, ++pos) {
      if (pos >= k.spike_cap) { set_error(k.status, FLYB_ETOOBIG, 5, s); break; }
      const int len = deg[q] - c < kEdgeChunk ? deg[q] - c : kEdgeChunk;
      k.spike_list[pos] = make_int4(bq[q], e0[q] + c, len, __float_as_int(xq[q]));
    }
  }
}

// Deferred delivery, scatter side: one block per list entry (at most kEdgeChunk edges), blocks
// striding over the entries the update kernel of step `s` appended; same integer red.global.add
// into the write slot as the fused path, so the ring sums are identical.
template <bool FIXED>
__global__ void __launch_bounds__(256) lif_scatter_kernel(LifK k, int s) {
  const Clk clk = read_clock(k);
  const int ws = slot_after(clk.ring_pos, s + k.n_delay, k.R);
  const size_t slot = (size_t)k.n * k.batch;
  const long long n = (long long)*k.spike_n < k.spike_cap ? (long long)*k.spike_n : k.spike_cap;
  unsigned long long edges = 0;
  for (long long j = blockIdx.x; j < n; j += gridDim.x) {
    const int4 en = k.spike_list[j];
    const float x = __int_as_float(en.w);
    for (int q = threadIdx.x; q < en.z; q += blockDim.x) {
      const int2 ed = __ldg(&k.out_edge[en.y + q]);
      const size_t dst = (size_t)ws * slot + (size_t)ed.x * k.batch + en.x;
      if (FIXED) {
        const long long f = __double2ll_rn((double)__int_as_float(ed.y) * (double)x * 4294967296.0);
        atomicAdd((unsigned long long*)k.ring + dst, (unsigned long long)f);
      } else {
        atomicAdd((int*)k.ring + dst, ed.y);
      }
    }
    edges += (unsigned long long)en.z;
  }
  if (k.events && threadIdx.x == 0 && edges) atomicAdd(k.events, edges);
}

// 32 x 32 bit transpose across a warp: lane r holds row r (bit c = column c) on entry and
// column r (bit c = row c) on return. Five exchanges: at distance j a lane keeps the half of each
// 2j-bit group on its own side and takes the partner's other half, rotated into place. The
// rotation and the kept bits depend only on the lane's side of each exchange, so they are
// computed once per thread. At distances 16 and 8 the halves are whole bytes, and one byte
// permute of (own word, partner's word) does the rotation and the merge: the lower side takes
// bytes {x0, x1, y0, y1} / {x0, y0, x2, y2}, the upper side {y2, y3, x2, x3} / {y1, x1, y3, x3}.
struct Transpose32 {
  int lane;
  __device__ __forceinline__ explicit Transpose32(int l) : lane(l) {}
  __device__ __forceinline__ unsigned operator()(unsigned x) const {
    constexpr unsigned M[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
    {
      const unsigned y = __shfl_xor_sync(0xffffffffu, x, 16);
      x = __byte_perm(x, y, (lane & 16) ? 0x3276u : 0x5410u);
    }
    {
      const unsigned y = __shfl_xor_sync(0xffffffffu, x, 8);
      x = __byte_perm(x, y, (lane & 8) ? 0x3715u : 0x6240u);
    }
#pragma unroll
    for (int q = 2; q < 5; ++q) {
      const int j = 16 >> q;
      const bool hi = lane & j;
      const unsigned y = __shfl_xor_sync(0xffffffffu, x, j);
      const unsigned t = __funnelshift_l(y, y, hi ? 32 - j : j);
      const unsigned keep = hi ? ~M[q] : M[q];
      x = (x & keep) | (t & ~keep);
    }
    return x;
  }
};

// Pull delivery (FLYB_LIF_PULL_DELIVERY) reads spike words from `pull_bits`, which the update
// kernels fill beside the spike history: the words of the last two groups of L consecutive steps,
// laid out [group parity][word][L], so one neuron's words of a whole group (G words per step, G =
// batch / 32) are G * L adjacent words. L = 8 / G makes that one 32-byte sector: the gather of an
// input then fetches every step of the group at once, where a per-step pull fetched a whole
// sector for G words of one step.
__device__ __forceinline__ size_t pull_word_index(const LifK& k, long long step, long long word) {
  const int sh = k.pull_group_log2;            // L is a power of two: shifts, no 64-bit division
  return (size_t)(((step >> sh) & 1) * k.words + word) * ((size_t)1 << sh) + (size_t)(step & ((1ll << sh) - 1));
}

// One input's words of a group: NW = G * L adjacent words (NW x 4-byte aligned).
template <int NW>
__device__ __forceinline__ void pull_words(const unsigned* __restrict__ bits, int pre, unsigned (&w)[NW]) {
  if (pre < 0) {
#pragma unroll
    for (int i = 0; i < NW; ++i) w[i] = 0u;
    return;
  }
  const unsigned* src = bits + (size_t)pre * NW;
  if constexpr (NW == 1) {
    w[0] = __ldg(src);
  } else if constexpr (NW == 2) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(src));
    w[0] = v.x; w[1] = v.y;
  } else if constexpr (NW == 8) {
    // the group's 32-byte sector in one 256-bit load (sm_100; `src` is 32-byte aligned)
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(src));
  } else {
#pragma unroll
    for (int i = 0; i < NW; i += 4) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + i));
      w[i] = v.x; w[i + 1] = v.y; w[i + 2] = v.z; w[i + 3] = v.w;
    }
  }
}

// The input tables stream through once per pull (cache-streaming loads), leaving L1 to the spike
// words the gathers reuse.
template <int P>
__device__ __forceinline__ void pull_planes(const unsigned* __restrict__ planes, long long c, unsigned (&pl)[P]) {
  const uint4* src = reinterpret_cast<const uint4*>(planes + (size_t)c * P);
#pragma unroll
  for (int q = 0; q < P; q += 4) {
    const uint4 v = __ldcs(src + q / 4);
    pl[q] = v.x; pl[q + 1] = v.y; pl[q + 2] = v.z; pl[q + 3] = v.w;
  }
}

// a mod m in [0, m) for any sign of a (m > 0).
__device__ __forceinline__ int pos_mod(long long a, int m) {
  const long long r = a % m;
  return (int)(r < 0 ? r + m : r);
}

// One chunk of a warp's input stream: every lane's G * L spike words of its input, the chunk's
// count planes (P of them from the plane table; P = 0: packed entries, the lane's own excess
// instead, from which the planes are rebuilt by ballots) and its base << 5 | plane count.
template <int NW, int P>
struct PullChunk {
  unsigned w[NW];
  unsigned pl[P > 0 ? P : 1];
  unsigned ex;
  int meta;
};

constexpr unsigned kPullPad = 0xFFFFFFu;        // packed entry: no input (a row's last chunk)

template <int NW, int P>
__device__ __forceinline__ void pull_fetch(const LifK& k, const unsigned* __restrict__ bits, int entry, long long c,
                                           PullChunk<NW, P>& x) {
  if constexpr (P == 0) {
    const unsigned pre = (unsigned)entry & kPullPad;
    pull_words<NW>(bits, pre == kPullPad ? -1 : (int)pre, x.w);
    x.ex = (unsigned)entry >> 24;
  } else {
    pull_words<NW>(bits, entry, x.w);
    pull_planes<P>(k.pull_planes, c, x.pl);
  }
  x.meta = __ldcs(&k.pull_meta[c]);
}

// The chunk's contribution for every step of the group: per step and fly group, the transposed
// mask m of the inputs that spiked and base x popc(m) + sum_{q < Q} 2^q popc(m & plane_q), Q the
// chunk's plane count as a template argument (chunk_sums dispatches on it once per chunk). Steps
// of the group outside the pull's range are summed too (one code path, no per-step tests) and
// never written.
template <int G, int L, int P, int Q>
__device__ __forceinline__ void chunk_sums_q(const Transpose32& transpose, const PullChunk<G * L, P>& x,
                                             int (&acc)[G * L]) {
  const int base = x.meta >> 5;
  unsigned pl[Q > 0 ? Q : 1];
#pragma unroll
  for (int q = 0; q < Q; ++q) pl[q] = P == 0 ? __ballot_sync(0xffffffffu, (x.ex >> q) & 1u) : x.pl[q];
#pragma unroll
  for (int u = 0; u < L; ++u) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const unsigned m = transpose(x.w[g * L + u]);
      int sum = base * __popc(m);
#pragma unroll
      for (int q = 0; q < Q; ++q) sum += __popc(m & pl[q]) << q;
      acc[g * L + u] += sum;
    }
  }
}

template <int G, int L, int P>
__device__ __forceinline__ void chunk_sums(const Transpose32& transpose, const PullChunk<G * L, P>& x,
                                           int (&acc)[G * L]) {
  constexpr int QMAX = P == 0 ? 8 : P;   // packed entries carry 8-bit excesses
#define FLYB_CHUNK(q) case q: chunk_sums_q<G, L, P, (q <= QMAX ? q : QMAX)>(transpose, x, acc); break;
  switch (x.meta & 31) {              // warp-uniform: one dispatch per chunk
    FLYB_CHUNK(0) FLYB_CHUNK(1) FLYB_CHUNK(2) FLYB_CHUNK(3) FLYB_CHUNK(4) FLYB_CHUNK(5) FLYB_CHUNK(6)
    FLYB_CHUNK(7) FLYB_CHUNK(8)
    default:
      if constexpr (P > 8) {
        switch (x.meta & 31) {
          FLYB_CHUNK(9) FLYB_CHUNK(10) FLYB_CHUNK(11) FLYB_CHUNK(12) FLYB_CHUNK(13) FLYB_CHUNK(14)
          FLYB_CHUNK(15) FLYB_CHUNK(16)
          default: break;
        }
      }
      break;
  }
#undef FLYB_CHUNK
}

// One warp's pass over postsynaptic rows [r0, r1) for the steps [lo, hi) of one group. The chunk
// stream is software-pipelined (the next chunk's words and the inputs of the one after are in
// flight while a chunk is summed); per chunk every step's words are transposed first and the plane
// sums of all of them are dispatched once on the chunk's plane count. A row's sums start from the
// values its write slots already hold, loaded when the row starts (their latency hides behind the
// row's first chunk), and are stored when it ends: the slots end with the same integers an add
// into them would leave, without a load waiting at the end of each row. Rows without inputs are
// not touched.
template <int G, int L, int P>
__device__ __forceinline__ void pull_pass(const LifK& k, const unsigned* __restrict__ bits, int r0, int r1, int lo,
                                          int hi, int ws0, int lane) {
  constexpr int NW = G * L;
  const Transpose32 transpose(lane);
  const size_t slot = (size_t)k.n * k.batch;
  const int ce = __ldg(&k.pull_ptr[r1]);
  int c = __ldg(&k.pull_ptr[r0]);
  if (c >= ce) return;                       // no row of the block has inputs
  int row = r0, bound = __ldg(&k.pull_ptr[r0 + 1]);
  int acc[NW];                               // [g * L + u], like the words
  const auto row_slot = [&](int u) {         // this lane's entry of `row` in the write slot of step u
    return (int*)k.ring + (size_t)slot_after(ws0, u, k.R) * slot + (size_t)row * k.batch + lane;
  };
  const auto start_row = [&]() {             // the first row at or after `row` that owns chunk c
    while (c >= bound) bound = __ldg(&k.pull_ptr[++row + 1]);
#pragma unroll
    for (int u = 0; u < L; ++u) {
      const bool on = u >= lo && u < hi;
      const int* src = on ? row_slot(u) : nullptr;
#pragma unroll
      for (int g = 0; g < G; ++g) acc[g * L + u] = on ? src[g * 32] : 0;
    }
  };
  const auto end_row = [&]() {               // the row's slots of steps [lo, hi) take the sums
#pragma unroll
    for (int u = 0; u < L; ++u) {
      if (u < lo || u >= hi) continue;
      int* dst = row_slot(u);
#pragma unroll
      for (int g = 0; g < G; ++g) dst[g * 32] = acc[g * L + u];
    }
  };
  PullChunk<NW, P> cur;
  pull_fetch<NW, P>(k, bits, __ldcs(&k.pull_pre[(size_t)c * 32 + lane]), c, cur);
  int pre_next = c + 1 < ce ? __ldcs(&k.pull_pre[(size_t)(c + 1) * 32 + lane]) : -1;
  start_row();
  for (; c < ce; ++c) {
    PullChunk<NW, P> nxt;
    int pre_after = -1;
    if (c + 1 < ce) {
      pull_fetch<NW, P>(k, bits, pre_next, c + 1, nxt);
      if (c + 2 < ce) pre_after = __ldcs(&k.pull_pre[(size_t)(c + 2) * 32 + lane]);
    }
    if (c >= bound) {                        // chunk c starts a later row: the current one is done
      end_row();
      start_row();
    }
    chunk_sums<G, L, P>(transpose, cur, acc);
    cur = nxt;
    pre_next = pre_after;
  }
  end_row();                                 // the last row with inputs
}

// Pull delivery of `nsteps` (1..L) undelivered steps, starting at pull_state[0] (its ring position
// pull_state[1]). Each warp owns a contiguous block of postsynaptic rows and walks their 32-input
// chunks as one stream, once per group of L steps the range touches (one group when the pulls
// follow the group ends, two when a range straddles a group end). Per chunk a lane gathers its
// input's G * L spike words of the group (one 32-byte sector); the warp transposes every word so
// that lane f holds, for fly f of a group of 32, the mask of the chunk's inputs that spiked, and
// adds base x popc(mask) + sum_p 2^p popc(mask & plane_p) (a row's inputs are sorted by count; a
// chunk stores its smallest count as the base and each entry's excess, packed into the entry's top
// byte or, for wide ranges, as up to 16 bit planes). Integer and exact: each step's write slot ends
// with the sums the scatter's atomics give. The chunk tables are read once per group instead of
// once per step. A row's sums start from its write slots' values and are stored back when the row
// ends, with coalesced 128-byte accesses per group of 32 flies. The synaptic events of presynaptic neurons in
// the warp's row block are counted from the same words. The last block to finish moves pull_state
// on by nsteps (every block has read it by then).
constexpr int kPullBlock = 256, kPullBlocksPerSm = 3;   // launch shape of the pull kernel
template <int G, int L, int P>
__global__ void __launch_bounds__(kPullBlock, kPullBlocksPerSm) lif_pull_kernel(LifK k, int nsteps) {
  constexpr int NW = G * L;
  const long long done = k.pull_state[0];
  const int rp_done = (int)k.pull_state[1];
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int per = (int)((k.n + warps - 1) / warps);
  const int r0 = (int)(wid * per < k.n ? wid * per : k.n);
  const int r1 = r0 + per < k.n ? r0 + per : k.n;
  unsigned long long ev = 0;
  const long long end = done + nsteps;
  for (long long grp = done / L; grp * L < end; ++grp) {
    const int lo = (int)((done > grp * L ? done : grp * L) - grp * L);          // steps [lo, hi) of the group
    const int hi = (int)((end < (grp + 1) * L ? end : (grp + 1) * L) - grp * L);
    const unsigned* __restrict__ bits = k.pull_bits + (size_t)(grp & 1) * k.words * L;
    // write slot of step grp * L + u: D slots after its read slot (consecutive steps, consecutive slots)
    const int ws0 = pos_mod(rp_done + (grp * L - done) + k.n_delay, k.R);
    if (r0 >= r1) continue;
    pull_pass<G, L, P>(k, bits, r0, r1, lo, hi, ws0, lane);
    if (k.events) {                          // events of presynaptic neurons r0 .. r1 in these steps
      for (int j = r0 + lane; j < r1; j += 32) {
        unsigned wj[NW];
        pull_words<NW>(bits, j, wj);
        int fl = 0;
#pragma unroll
        for (int u = 0; u < L; ++u) {
          if (u < lo || u >= hi) continue;
#pragma unroll
          for (int g = 0; g < G; ++g) fl += __popc(wj[g * L + u]);
        }
        if (fl) ev += (unsigned long long)fl * (unsigned)(__ldg(&k.out_ptr[j + 1]) - __ldg(&k.out_ptr[j]));
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ev += __shfl_xor_sync(0xffffffffu, ev, o);
  if (k.events && lane == 0 && ev) atomicAdd(k.events, ev);
  // the last block to finish moves the undelivered range on (every block read it at its start)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned long long prev = atomicAdd(reinterpret_cast<unsigned long long*>(k.pull_state + 2), 1ull);
    if (prev == (unsigned long long)gridDim.x - 1) {
      k.pull_state[0] = end;
      k.pull_state[1] = pos_mod(rp_done + nsteps, k.R);
      k.pull_state[2] = 0;
      __threadfence();
    }
  }
}

// The pull kernel uses no shared memory: it asks for the largest L1, where part of the spike words
// its gathers read stays resident, and runs as one wave of resident blocks.
template <int G, int L, int P>
static void launch_pull_glp(const LifK& k, int nsteps, int sms, cudaStream_t st) {
  static int per_sm = 0;                 // resident blocks: one wave, each warp a longer row stream
  if (!per_sm) {
    cudaFuncSetAttribute(lif_pull_kernel<G, L, P>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lif_pull_kernel<G, L, P>, kPullBlock, 0);
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = k.pull_grid > 0 && k.pull_grid < sms * per_sm ? k.pull_grid : sms * per_sm;
  lif_pull_kernel<G, L, P><<<grid, kPullBlock, 0, st>>>(k, nsteps);
}

template <int G, int L>
static void launch_pull_gl(const LifK& k, int nsteps, int sms, cudaStream_t st) {
  if (k.pull_nplanes == 0) launch_pull_glp<G, L, 0>(k, nsteps, sms, st);
  else launch_pull_glp<G, L, 16>(k, nsteps, sms, st);
}

// Steps per group a batch width allows: 8 / G (one sector per input and group), or 1.
static bool pull_group_ok(int batch, int L) {
  const int g = batch / 32;
  return L == 1 || L == 8 / g;
}

static int launch_pull(const LifK& k, int nsteps, cudaStream_t st) {
  if (nsteps < 1 || nsteps > k.pull_group) return FLYB_EINVAL;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool grouped = k.pull_group > 1;
  switch (k.batch / 32) {
    case 1: grouped ? launch_pull_gl<1, 8>(k, nsteps, sms, st) : launch_pull_gl<1, 1>(k, nsteps, sms, st); break;
    case 2: grouped ? launch_pull_gl<2, 4>(k, nsteps, sms, st) : launch_pull_gl<2, 1>(k, nsteps, sms, st); break;
    case 4: grouped ? launch_pull_gl<4, 2>(k, nsteps, sms, st) : launch_pull_gl<4, 1>(k, nsteps, sms, st); break;
    case 8: launch_pull_gl<8, 1>(k, nsteps, sms, st); break;
    default: return FLYB_EINVAL;
  }
  return (int)cudaGetLastError();
}

// Whether the launch pulls its steps itself: pull delivery over all neurons.
static bool pulls_itself(const LifK& k) {
  return (k.flags & FLYB_LIF_PULL_DELIVERY) && k.t_begin == 0 && k.t_end == (long long)k.n * k.batch;
}

// A run that pulls itself delivers at every group end (local step s ends a group when the step
// index, pull_phase + s + 1 counted from a group start, is a multiple of L) and after its last
// step, so it ends with nothing pending. `pending` counts the steps since the last pull.
static int pull_after_step(const LifK& k, int s, int& pending, cudaStream_t st) {
  if (!pulls_itself(k)) return 0;
  ++pending;
  if ((k.pull_phase + s + 1) % k.pull_group != 0 && s != k.nsteps - 1) return 0;
  const int rc = launch_pull(k, pending, st);
  pending = 0;
  return rc;
}

// One block processes work items [base, base + BLOCK*IPT) of local step `s`: update, then deliver.
// Thread j owns the IPT consecutive items base + j*IPT + q (neuron-major, fly-minor order), loads
// every state array as one vector and keeps all loads in flight before computing.
template <int BLOCK, bool FIXED, int IPT, bool DEFER = false>
__device__ __forceinline__ void lif_chunk(const LifK& k, const Clk& clk, int s, long long base,
                                          LifSmem<BLOCK * IPT>& sm) {
  using RingT = typename std::conditional<FIXED, long long, int>::type;
  const long long W = k.t_end;                         // items of this launch end here
  const long long t0 = base + (long long)threadIdx.x * IPT;
  const int rs = slot_after(clk.ring_pos, s, k.R);
  const int ws = slot_after(clk.ring_pos, s + k.n_delay, k.R);
  const size_t slot = (size_t)k.n * k.batch;            // ring slot stride
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const LifP& P = k.P;
  const int flags = k.flags;
  unsigned fired_bits = 0, tx_bits = 0;
  float xq[IPT];
  int iq[IPT], bq[IPT];
#pragma unroll
  for (int q = 0; q < IPT; ++q) { xq[q] = 0.0f; iq[q] = 0; bq[q] = 0; }
  if (t0 < W) {
    const bool whole = t0 + IPT <= W;   // every item of the vector exists (the tail is done by items)
    RingT c[IPT];
    float vv[IPT], gg[IPT], ref[IPT], ad[IPT], dv[IPT], pp[IPT], rt[IPT], cn[IPT], rr[IPT];
    RingT* rp = (RingT*)k.ring + (size_t)rs * slot + t0;
    if (whole) {
      vload<IPT>(rp, c);
      vload<IPT>(k.v + t0, vv); vload<IPT>(k.g + t0, gg); vload<IPT>(k.refrac + t0, ref);
      vload<IPT>(k.adapt + t0, ad); vload<IPT>(k.drive + t0, dv); vload<IPT>(k.rate + t0, rt);
      if (flags & FLYB_LIF_POISSON) vload<IPT>(k.poisson_p + t0, pp);
      if (flags & FLYB_LIF_COUNTS) vload<IPT>(k.counts + t0, cn);
      if (flags & FLYB_LIF_STD) vload<IPT>(k.res + t0, rr);
    } else {
#pragma unroll
      for (int q = 0; q < IPT; ++q) {
        const bool ok = t0 + q < W;
        c[q] = ok ? rp[q] : 0;
        vv[q] = ok ? k.v[t0 + q] : 0.0f; gg[q] = ok ? k.g[t0 + q] : 0.0f; ref[q] = ok ? k.refrac[t0 + q] : 0.0f;
        ad[q] = ok ? k.adapt[t0 + q] : 0.0f; dv[q] = ok ? k.drive[t0 + q] : 0.0f; rt[q] = ok ? k.rate[t0 + q] : 0.0f;
        pp[q] = (ok && (flags & FLYB_LIF_POISSON)) ? k.poisson_p[t0 + q] : 0.0f;
        cn[q] = (ok && (flags & FLYB_LIF_COUNTS)) ? k.counts[t0 + q] : 0.0f;
        rr[q] = (ok && (flags & FLYB_LIF_STD)) ? k.res[t0 + q] : 1.0f;
      }
    }
    if (!(flags & FLYB_LIF_POISSON)) {
#pragma unroll
      for (int q = 0; q < IPT; ++q) pp[q] = 0.0f;
    }
    RingT nc[IPT];
    float sp[IPT];
    bool touched = false;
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const long long t = t0 + q;
      nc[q] = c[q];
      sp[q] = 0.0f;
      if (t >= W) continue;
      // the fused path keeps the 64-bit division: its register allocation (and occupancy) depends
      // on it; the deferred path divides by multiply-shift
      const int i = DEFER ? neuron_of(k, (int)t) : (int)(t / k.batch);
      const int b = DEFER ? (int)t - i * k.batch : (int)(t - (long long)i * k.batch);
      iq[q] = i;
      bq[q] = b;
      const bool live = !(flags & FLYB_LIF_EPISODES) || s < k.fly_steps[b];
      if (!live) { sp[q] = k.spikes[t]; continue; }
      nc[q] = 0;
      const float act = k.active[i];
      bool skip = false;
      if ((flags & FLYB_LIF_SKIP_FROZEN) && act == 0.0f && pp[q] == 0.0f && c[q] == 0) {
        // frozen cell at rest: the update would leave it unchanged (neural.cu:24-26)
        const float rres = (flags & FLYB_LIF_STD) ? rr[q] : k.res[t];
        skip = vv[q] == P.v_rest && gg[q] == 0.0f && dv[q] == 0.0f && ad[q] == 0.0f && ref[q] == 0.0f &&
               rt[q] == 0.0f && k.spikes[t] == 0.0f && rres == 1.0f;
      }
      if (skip) continue;           // sp stays 0 == the cell's spike value
      touched = true;
      // steps 1-4, the arithmetic of lif_update written out over the item vectors (kept inline: the
      // vector path's register allocation, and with it its occupancy, depends on it)
      // 1. synaptic input due now
      float g1 = gg[q] * P.a_s;
      if (c[q]) {
        const float inc = FIXED ? __double2float_rn((double)c[q] * (1.0 / 4294967296.0)) : P.w_syn * (float)c[q];
        g1 = g1 + inc;
      }
      gg[q] = g1;
      // 2. membrane, exponential Euler with g and drive held (brain.py:839-843)
      float target = P.v_rest + g1;
      target = target + dv[q];
      target = target - ad[q];
      float u = vv[q] - target;
      u = u * P.a_m;
      float v1 = target + u;
      float r1 = ref[q];
      if (r1 > 0.0f) v1 = P.v_reset;
      r1 = r1 - P.dt;
      if (r1 < 0.0f) r1 = 0.0f;
      // 3. threshold x active, Poisson forcing (brain.py:845-849)
      float spike = (v1 >= P.v_th ? 1.0f : 0.0f) * act;
      if (pp[q] > 0.0f) {
        const float un = (flags & FLYB_LIF_EXT_UNIFORM)
                             ? k.uniforms[(size_t)s * slot + t]
                             : philox_uniform(k.seed, clk.step0 + s, (uint32_t)i, (uint32_t)(k.fly0 + b));
        if (un < pp[q]) spike = 1.0f;
      }
      const bool fired = spike > 0.0f;
      if (fired) { v1 = P.v_reset; r1 = P.t_ref; }
      vv[q] = v1;
      ref[q] = r1;
      sp[q] = spike;
      // 4. adaptation, depression, counters, rate (brain.py:853-868)
      if (flags & FLYB_LIF_ADAPT) {
        float a1 = ad[q] * P.a_ad;
        a1 = a1 + spike * (k.adapt_jump ? __ldg(&k.adapt_jump[i]) : P.jump);
        ad[q] = a1;
      }
      float x = spike;
      if (flags & FLYB_LIF_STD) {
        float r2 = rr[q];
        x = spike * r2;
        if (fired) { const float keep = 1.0f - k.std_u[i]; r2 = r2 * keep; }
        float dep = 1.0f - r2;
        dep = dep * P.a_std;
        rr[q] = 1.0f - dep;
      }
      if (flags & FLYB_LIF_COUNTS) cn[q] = cn[q] + spike;
      float r3 = rt[q] * P.a_r;
      r3 = r3 + spike * P.rg;
      rt[q] = r3;
      if (fired) fired_bits |= 1u << q;
      if (x != 0.0f) { tx_bits |= 1u << q; xq[q] = x; }
    }
    bool ring_changed = false;
#pragma unroll
    for (int q = 0; q < IPT; ++q) ring_changed |= nc[q] != c[q];
    if (whole) {
      if (ring_changed) vstore<IPT>(rp, nc);
      if (touched) {
        vstore<IPT>(k.g + t0, gg); vstore<IPT>(k.v + t0, vv); vstore<IPT>(k.refrac + t0, ref);
        vstore<IPT>(k.spikes + t0, sp); vstore<IPT>(k.rate + t0, rt);
        if (flags & FLYB_LIF_ADAPT) vstore<IPT>(k.adapt + t0, ad);
        if (flags & FLYB_LIF_STD) vstore<IPT>(k.res + t0, rr);
        if (flags & FLYB_LIF_COUNTS) vstore<IPT>(k.counts + t0, cn);
      }
    } else {
#pragma unroll
      for (int q = 0; q < IPT; ++q) {
        if (t0 + q >= W) continue;
        const long long t = t0 + q;
        if (nc[q] != c[q]) rp[q] = nc[q];
        if (touched) {
          k.g[t] = gg[q]; k.v[t] = vv[q]; k.refrac[t] = ref[q]; k.spikes[t] = sp[q]; k.rate[t] = rt[q];
          if (flags & FLYB_LIF_ADAPT) k.adapt[t] = ad[q];
          if (flags & FLYB_LIF_STD) k.res[t] = rr[q];
          if (flags & FLYB_LIF_COUNTS) k.counts[t] = cn[q];
        }
      }
    }
  }
  // raster words: a warp covers 32 * IPT items = IPT words; lane l's IPT bits go to word l / (32/IPT)
  if (k.raster) {
    constexpr int LPW = 32 / IPT;            // lanes per raster word
    unsigned v = fired_bits << (IPT * (lane % LPW));
#pragma unroll
    for (int o = 1; o < LPW; o <<= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    const long long wbase = base + (long long)warp * 32 * IPT;
    if (lane % LPW == 0 && wbase + (long long)(lane / LPW) * 32 < W) {
      const size_t rslot = k.raster_slots > 0 ? (size_t)slot_after(clk.raster_pos, s, k.raster_slots) : (size_t)s;
      k.raster[rslot * k.words + (size_t)((wbase >> 5) + lane / LPW)] = v;
      if (k.pull_bits) k.pull_bits[pull_word_index(k, clk.step0 + s, (wbase >> 5) + lane / LPW)] = v;
    }
  }
  if constexpr (DEFER)
    append_spikes<IPT>(k, s, tx_bits, iq, bq, xq);
  else if (!(k.flags & FLYB_LIF_PULL_DELIVERY))
    deliver<BLOCK, FIXED, IPT>(k, sm, tx_bits, iq, bq, xq, ws, slot);
}

// The deferred-delivery update at 1-2 items per thread is bounded to 64 registers (32 warps per SM
// stay resident; at 4 items the bound would spill).
template <int BLOCK, bool FIXED, int IPT, bool DEFER = false>
__global__ void __launch_bounds__(BLOCK, (DEFER && IPT <= 2) ? 1024 / BLOCK : 1) lif_step_kernel(LifK k, int s) {
  __shared__ LifSmem<BLOCK * IPT> sm;
  const Clk clk = read_clock(k);
  lif_chunk<BLOCK, FIXED, IPT, DEFER>(k, clk, s, k.t_begin + (long long)blockIdx.x * BLOCK * IPT, sm);
}

__global__ void lif_advance_kernel(LifK k) { advance_clock(k, read_clock(k)); }

// ------------------------------------------------------------------ clocks and the slow tone
// The clocked step (brain.py:899-957): neuron i updates on steps with step % k_i == 0, with the
// coefficients of a k_i * dt step (row k_i of clock_coef); on other steps it takes row 0 (no
// decay, no refractory time, no spike, no Poisson). Input arriving at a period-k_i neuron between
// its updates is summed exactly in clock_acc and applied on the update step, as the reference
// applies W_k to the spikes accumulated over the period.
// The slow tone (brain.py:551-585, 829-845): per class, the tone decays and takes its delayed
// input from its own exact ring; the summed tone joins the membrane target, scales the fast input
// or lowers the threshold. Its spikes go out on each class's synapse list after the fast ones.
// Under clocks a class decays by its column of the phase row and its input to a period-k neuron
// waits for the update like the fast input (brain.py:905-917).
// One item per thread, then the block-wide delivery of the register path.
// Input reaching a neuron that updates every `period` > 1 steps: summed exactly in *acc while the
// neuron holds, returned whole (with this step's) on its update step.
__device__ __forceinline__ long long hold_until_update(long long* acc, long long due, bool on) {
  const long long held = *acc, sum = held + due;
  const long long keep = on ? 0 : sum;
  if (keep != held) *acc = keep;
  return on ? sum : 0;
}

template <int BLOCK, bool FIXED>
__global__ void __launch_bounds__(BLOCK) lif_ext_kernel(LifK k, int s) {
  using RingT = typename std::conditional<FIXED, long long, int>::type;
  __shared__ LifSmem<BLOCK> sm;
  const Clk clk = read_clock(k);
  const long long W = k.t_end;
  const long long t = k.t_begin + (long long)blockIdx.x * BLOCK + threadIdx.x;
  const int rs = slot_after(clk.ring_pos, s, k.R);
  const int ws = slot_after(clk.ring_pos, s + k.n_delay, k.R);
  const size_t slot = (size_t)k.n * k.batch;
  const int flags = k.flags;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const LifP& P = k.P;
  unsigned fired_bit = 0, tx_bit = 0;
  int iq[1] = {0}, bq[1] = {0};
  float xq[1] = {0.0f};
  if (t < W) {
    const int i = (int)(t / k.batch), b = (int)(t - (long long)i * k.batch);
    iq[0] = i;
    bq[0] = b;
    const bool live = !(flags & FLYB_LIF_EPISODES) || s < k.fly_steps[b];
    if (live) {
      RingT* rp = (RingT*)k.ring + (size_t)rs * slot + t;
      long long due = *rp;
      if (due) *rp = 0;
      // this step's coefficients: the neuron's phase row under clocks, else the step's own
      float c_m = P.a_m, c_s = P.a_s, c_dt = P.dt, c_ad = P.a_ad, c_std = P.a_std, c_r = P.a_r, c_rg = P.rg;
      float c_u = 1.0f, c_pois = 1.0f;
      const float* cf = nullptr;   // the phase row under clocks
      int period = 1;
      bool on = true;
      if (k.clock_k) {
        const long long step = clk.step0 + s;
        period = k.clock_k[i];
        on = period == 1 || step % period == 0;
        if (period > 1) due = hold_until_update(k.clock_acc + t, due, on);
        cf = k.clock_coef + FLYB_CLOCK_NCOEF * (on ? period : 0);
        c_m = cf[FLYB_CLOCK_A_M], c_s = cf[FLYB_CLOCK_A_S], c_dt = cf[FLYB_CLOCK_DT], c_ad = cf[FLYB_CLOCK_A_AD];
        c_std = cf[FLYB_CLOCK_A_STD], c_r = cf[FLYB_CLOCK_A_R], c_rg = cf[FLYB_CLOCK_RATE_GAIN];
        c_u = cf[FLYB_CLOCK_U], c_pois = cf[FLYB_CLOCK_POIS];
      }
      const float act = k.active[i];
      float g1 = k.g[t] * c_s;
      if (due) {
        const float inc = FIXED ? __double2float_rn((double)due * (1.0 / 4294967296.0)) : P.w_syn * (float)due;
        g1 = g1 + inc;
      }
      k.g[t] = g1;
      // slow tone: each class decays and takes its delayed input; the classes are summed in order
      float tone = 0.0f;
      for (int c = 0; c < k.slow_classes; ++c) {
        long long* sp = k.slow_ring[c] + (size_t)rs * slot + t;
        long long sdue = *sp;
        if (sdue) *sp = 0;
        if (period > 1) sdue = hold_until_update(k.slow_clock_acc[c] + t, sdue, on);
        float sg = k.slow_g[c][t] * (cf ? cf[FLYB_CLOCK_A_SLOW0 + c] : k.slow_decay[c]);
        if (sdue) sg = sg + __double2float_rn((double)sdue * (1.0 / 4294967296.0));
        k.slow_g[c][t] = sg;
        tone = tone + sg;
      }
      if (k.slow_classes) k.g_slow[t] = tone;
      const float ad = k.adapt[t];
      float th = P.v_th;
      float target;
      if (k.slow_classes && k.slow_mode == FLYB_SLOW_GAIN) {
        float f = 1.0f + tone / k.slow_norm;
        f = fminf(fmaxf(f, k.slow_clip_lo), k.slow_clip_hi);
        target = P.v_rest + g1 * f;
      } else {
        target = P.v_rest + g1;
      }
      target = target + k.drive[t];
      target = target - ad;
      if (k.slow_classes && k.slow_mode == FLYB_SLOW_ADDITIVE) target = target + tone;
      if (k.slow_classes && k.slow_mode == FLYB_SLOW_THRESHOLD) th = -fminf(tone, k.slow_th_max) + P.v_th;
      float u = k.v[t] - target;
      u = u * c_m;
      float v1 = target + u;
      float r1 = k.refrac[t];
      if (r1 > 0.0f) v1 = P.v_reset;
      r1 = r1 - c_dt;
      if (r1 < 0.0f) r1 = 0.0f;
      float spike = (v1 >= th ? 1.0f : 0.0f) * c_u;
      spike = spike * act;
      if (flags & FLYB_LIF_POISSON) {
        const float q = k.poisson_p[t] * c_pois;
        if (q > 0.0f) {
          const float un = (flags & FLYB_LIF_EXT_UNIFORM)
                               ? k.uniforms[(size_t)s * slot + t]
                               : philox_uniform(k.seed, clk.step0 + s, (uint32_t)i, (uint32_t)(k.fly0 + b));
          if (un < q) spike = 1.0f;
        }
      }
      const bool fired = spike > 0.0f;
      if (fired) { v1 = P.v_reset; r1 = P.t_ref; }
      k.v[t] = v1;
      k.refrac[t] = r1;
      k.spikes[t] = spike;
      if (flags & FLYB_LIF_ADAPT) {
        float a1 = ad * c_ad;
        a1 = a1 + spike * (k.adapt_jump ? __ldg(&k.adapt_jump[i]) : P.jump);
        k.adapt[t] = a1;
      }
      float x = spike;
      if (flags & FLYB_LIF_STD) {
        float r2 = k.res[t];
        x = spike * r2;
        if (fired) { const float keep = 1.0f - k.std_u[i]; r2 = r2 * keep; }
        float dep = 1.0f - r2;
        dep = dep * c_std;
        k.res[t] = 1.0f - dep;
      }
      if (flags & FLYB_LIF_COUNTS) k.counts[t] = k.counts[t] + spike;
      float r3 = k.rate[t] * c_r;
      r3 = r3 + spike * c_rg;
      k.rate[t] = r3;
      if (fired) fired_bit = 1u;
      if (x != 0.0f) { tx_bit = 1u; xq[0] = x; }
    }
  }
  if (k.raster) {
    const unsigned bits = __ballot_sync(0xffffffffu, fired_bit);
    const long long wbase = k.t_begin + (long long)blockIdx.x * BLOCK + (long long)warp * 32;
    if (lane == 0 && wbase < W) {
      const size_t rslot = k.raster_slots > 0 ? (size_t)slot_after(clk.raster_pos, s, k.raster_slots) : (size_t)s;
      k.raster[rslot * k.words + (size_t)(wbase >> 5)] = bits;
    }
  }
  deliver<BLOCK, FIXED, 1>(k, sm, tx_bit, iq, bq, xq, ws, slot);
  for (int c = 0; c < k.slow_classes; ++c) {     // the same transmitted amounts onto each slow list
    LifK ks = k;
    ks.out_ptr = k.slow_out_ptr[c];
    ks.out_edge = k.slow_out_edge[c];
    ks.ring = k.slow_ring[c];
    ks.events = nullptr;
    deliver<BLOCK, true, 1>(ks, sm, tx_bit, iq, bq, xq, ws, slot);
  }
}

static bool needs_advance(const LifK& k);

template <int BLOCK, bool FIXED>
static int run_lif_ext(const LifK& k, cudaStream_t st) {
  const long long W = (long long)k.t_end - k.t_begin;
  const unsigned blocks = (unsigned)((W + BLOCK - 1) / BLOCK);
  for (int s = 0; s < k.nsteps; ++s) {
    lif_ext_kernel<BLOCK, FIXED><<<blocks, BLOCK, 0, st>>>(k, s);
    FLYB_CHECK_LAUNCH();
  }
  if (needs_advance(k)) {
    lif_advance_kernel<<<1, 256, 0, st>>>(k);
    FLYB_CHECK_LAUNCH();
  }
  return 0;
}

// A run ends by advancing the device clock / episode counters unless the caller does it later.
static bool needs_advance(const LifK& k) {
  return (k.clock || (k.flags & FLYB_LIF_EPISODES)) && !(k.flags & FLYB_LIF_NO_ADVANCE);
}

template <int BLOCK, bool FIXED, int IPT>
__global__ void __launch_bounds__(BLOCK) lif_persistent_kernel(LifK k) {
  __shared__ LifSmem<BLOCK * IPT> sm;
  const Clk clk = read_clock(k);
  int generation = 0;
  for (int s = 0; s < k.nsteps; ++s) {
    for (long long base = k.t_begin + (long long)blockIdx.x * BLOCK * IPT; base < k.t_end;
         base += (long long)gridDim.x * BLOCK * IPT)
      lif_chunk<BLOCK, FIXED, IPT>(k, clk, s, base, sm);
    // the next step writes the slot this step read: every block must be done with it
    if (!grid_barrier(k.sync, k.status, generation, s)) return;
  }
  // every block has read the clock and the episode counters: advance them
  if (blockIdx.x == 0 && !(k.flags & FLYB_LIF_NO_ADVANCE)) advance_clock(k, clk);
}

// ------------------------------------------------------------------ staged (bulk-copy) step
// One step, per-step launch, blocks looping over chunks of CH = BLOCK * IPT items. A chunk's state
// arrays are copied global -> shared by the async proxy (cp.async.bulk, completion on an mbarrier)
// while the block updates and delivers the previous chunk from the other stage; the updated arrays
// go back shared -> global the same way. Thread j handles items j + r * BLOCK of a chunk (r < IPT),
// one at a time from shared memory, so the registers hold one item and the copies in flight
// replace the vector loads of the register path.
template <int BLOCK, bool FIXED, int IPT>
struct StagedLayout {
  using RingT = typename std::conditional<FIXED, long long, int>::type;
  static constexpr int CH = BLOCK * IPT;
  enum { V, G, REF, AD, DV, RT, PP, CN, RR, NF };             // float arrays of a stage; DV holds spikes out
  static constexpr size_t RING = (size_t)CH * sizeof(RingT);
  static constexpr size_t STAGE = RING + (size_t)NF * CH * sizeof(float);
  static constexpr size_t BARS = 128;                          // two mbarriers, padded
  static constexpr size_t LISTS = BARS + 2 * STAGE;
  static constexpr size_t BYTES = LISTS + sizeof(LifSmem<CH>);
};

// Loads of the chunk starting at item `base` (items up to W) into `stage`, on barrier `bar`.
template <int BLOCK, bool FIXED, int IPT>
__device__ __forceinline__ void staged_issue_loads(const LifK& k, unsigned char* stage, long long base, long long W,
                                                   const void* ring_rd, uint64_t* bar) {
  using L = StagedLayout<BLOCK, FIXED, IPT>;
  using RingT = typename L::RingT;
  const long long n = W - base < L::CH ? W - base : L::CH;      // a multiple of 4 (checked on the host)
  const uint32_t fb = (uint32_t)(n * sizeof(float)), rb = (uint32_t)(n * sizeof(RingT));
  float* f = reinterpret_cast<float*>(stage + L::RING);
  const int flags = k.flags;
  const int nf = 6 + ((flags & FLYB_LIF_POISSON) ? 1 : 0) + ((flags & FLYB_LIF_COUNTS) ? 1 : 0) +
                 ((flags & FLYB_LIF_STD) ? 1 : 0);
  mbar_arrive_expect(bar, rb + (uint32_t)nf * fb);
  bulk_load(stage, (const RingT*)ring_rd + base, rb, bar);
  bulk_load(f + L::V * L::CH, k.v + base, fb, bar);
  bulk_load(f + L::G * L::CH, k.g + base, fb, bar);
  bulk_load(f + L::REF * L::CH, k.refrac + base, fb, bar);
  bulk_load(f + L::AD * L::CH, k.adapt + base, fb, bar);
  bulk_load(f + L::DV * L::CH, k.drive + base, fb, bar);
  bulk_load(f + L::RT * L::CH, k.rate + base, fb, bar);
  if (flags & FLYB_LIF_POISSON) bulk_load(f + L::PP * L::CH, k.poisson_p + base, fb, bar);
  if (flags & FLYB_LIF_COUNTS) bulk_load(f + L::CN * L::CH, k.counts + base, fb, bar);
  if (flags & FLYB_LIF_STD) bulk_load(f + L::RR * L::CH, k.res + base, fb, bar);
}

template <int BLOCK, bool FIXED, int IPT>
__device__ __forceinline__ void staged_issue_stores(const LifK& k, unsigned char* stage, long long base, long long W) {
  using L = StagedLayout<BLOCK, FIXED, IPT>;
  const long long n = W - base < L::CH ? W - base : L::CH;
  const uint32_t fb = (uint32_t)(n * sizeof(float));
  float* f = reinterpret_cast<float*>(stage + L::RING);
  const int flags = k.flags;
  bulk_store(k.v + base, f + L::V * L::CH, fb);
  bulk_store(k.g + base, f + L::G * L::CH, fb);
  bulk_store(k.refrac + base, f + L::REF * L::CH, fb);
  bulk_store(k.spikes + base, f + L::DV * L::CH, fb);
  bulk_store(k.rate + base, f + L::RT * L::CH, fb);
  if (flags & FLYB_LIF_ADAPT) bulk_store(k.adapt + base, f + L::AD * L::CH, fb);
  if (flags & FLYB_LIF_COUNTS) bulk_store(k.counts + base, f + L::CN * L::CH, fb);
  if (flags & FLYB_LIF_STD) bulk_store(k.res + base, f + L::RR * L::CH, fb);
  bulk_commit();
}

template <int BLOCK, bool FIXED, int IPT, bool DEFER = false>
__global__ void __launch_bounds__(BLOCK) lif_staged_kernel(LifK k, int s) {
  using L = StagedLayout<BLOCK, FIXED, IPT>;
  using RingT = typename L::RingT;
  constexpr int CH = L::CH;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  LifSmem<CH>& sm = *reinterpret_cast<LifSmem<CH>*>(smem + L::LISTS);
  __shared__ int ok;
  const long long W = k.t_end;                                 // items [t_begin, t_end) of this launch
  const long long nchunks = (W - k.t_begin + CH - 1) / CH;
  const size_t slot = (size_t)k.n * k.batch;                  // ring slot stride
  if ((long long)blockIdx.x >= nchunks) return;                 // block-uniform, before any copy
  const Clk clk = read_clock(k);
  const int rs = slot_after(clk.ring_pos, s, k.R);
  const int ws = slot_after(clk.ring_pos, s + k.n_delay, k.R);
  RingT* ring_rd = (RingT*)k.ring + (size_t)rs * slot;
  const LifP& P = k.P;
  const int flags = k.flags;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    staged_issue_loads<BLOCK, FIXED, IPT>(k, smem + L::BARS, k.t_begin + (long long)blockIdx.x * CH, W, ring_rd,
                                          &bar[0]);
  }
  uint32_t parity = 0u;                                        // bit st: phase parity of stage st
  int it = 0;
  for (long long c = blockIdx.x; c < nchunks; c += gridDim.x, ++it) {
    const int st = it & 1;
    unsigned char* stage = smem + L::BARS + (size_t)st * L::STAGE;
    const long long base = k.t_begin + c * CH;
    if (threadIdx.x == 0) {
      const long long cn = c + gridDim.x;
      if (cn < nchunks) {
        bulk_wait_read_all();     // the other stage's stores (previous chunk) have read it out
        staged_issue_loads<BLOCK, FIXED, IPT>(k, smem + L::BARS + (size_t)(st ^ 1) * L::STAGE, k.t_begin + cn * CH,
                                              W, ring_rd, &bar[st ^ 1]);
      }
      ok = mbar_wait_bounded(&bar[st], (parity >> st) & 1u, k.status, kMbarLimit, 4, s) ? 1 : 0;
      // on a timeout, let this block's other copy in flight land before it leaves
      if (!ok && cn < nchunks) mbar_wait_bounded(&bar[st ^ 1], (parity >> (st ^ 1)) & 1u, k.status, kMbarLimit, 4, s);
    }
    __syncthreads();
    if (!ok) {
      if (threadIdx.x == 0) bulk_wait_all();
      return;
    }
    mbar_try_wait(&bar[st], (parity >> st) & 1u);   // completed: each thread observes the phase (acquire)
    parity ^= 1u << st;
    RingT* ring = reinterpret_cast<RingT*>(stage);
    float* f = reinterpret_cast<float*>(stage + L::RING);
    unsigned tx_bits = 0;
    float xq[IPT];
    int iq[IPT], bq[IPT];
#pragma unroll
    for (int r = 0; r < IPT; ++r) {
      const int j = threadIdx.x + r * BLOCK;
      const int t = (int)base + j;                              // n * batch < 2^31
      bool fired = false;
      xq[r] = 0.0f; iq[r] = 0; bq[r] = 0;
      if (t < W) {
        const int i = neuron_of(k, t), b = t - i * k.batch;
        iq[r] = i;
        bq[r] = b;
        const RingT c0 = ring[j];
        const bool live = !(flags & FLYB_LIF_EPISODES) || s < k.fly_steps[b];
        if (!live) {
          f[L::DV * CH + j] = k.spikes[t];                      // unchanged state, spike kept
        } else {
          if (c0) ring_rd[t] = 0;
          float vv = f[L::V * CH + j], gg = f[L::G * CH + j], ref = f[L::REF * CH + j], ad = f[L::AD * CH + j];
          const float dv = f[L::DV * CH + j];
          float rt = f[L::RT * CH + j];
          const float pp = (flags & FLYB_LIF_POISSON) ? f[L::PP * CH + j] : 0.0f;
          float cn = (flags & FLYB_LIF_COUNTS) ? f[L::CN * CH + j] : 0.0f;
          float rr = (flags & FLYB_LIF_STD) ? f[L::RR * CH + j] : 1.0f;
          const float act = k.active[i];
          bool skip = false;
          if ((flags & FLYB_LIF_SKIP_FROZEN) && act == 0.0f && pp == 0.0f && c0 == 0) {
            const float rres = (flags & FLYB_LIF_STD) ? rr : k.res[t];
            skip = vv == P.v_rest && gg == 0.0f && dv == 0.0f && ad == 0.0f && ref == 0.0f && rt == 0.0f &&
                   k.spikes[t] == 0.0f && rres == 1.0f;
          }
          if (skip) {
            f[L::DV * CH + j] = 0.0f;
          } else {
            float x;
            const float spike = lif_update<FIXED>(k, clk, s, slot, (size_t)t, i, b, c0, act, pp, dv, vv, gg, ref, ad,
                                                  rt, cn, rr, x);
            fired = spike > 0.0f;
            f[L::V * CH + j] = vv; f[L::G * CH + j] = gg; f[L::REF * CH + j] = ref; f[L::AD * CH + j] = ad;
            f[L::DV * CH + j] = spike; f[L::RT * CH + j] = rt;
            if (flags & FLYB_LIF_COUNTS) f[L::CN * CH + j] = cn;
            if (flags & FLYB_LIF_STD) f[L::RR * CH + j] = rr;
            if (x != 0.0f) { tx_bits |= 1u << r; xq[r] = x; }
          }
        }
      }
      // raster: lanes of a warp hold 32 consecutive items of the chunk = one word
      if (k.raster) {
        const unsigned word = __ballot_sync(0xffffffffu, fired);
        const int wfirst = (int)base + r * BLOCK + warp * 32;
        if (lane == 0 && wfirst < W) {
          const size_t rslot = k.raster_slots > 0 ? (size_t)slot_after(clk.raster_pos, s, k.raster_slots) : (size_t)s;
          k.raster[rslot * k.words + (size_t)(wfirst >> 5)] = word;
          if (k.pull_bits) k.pull_bits[pull_word_index(k, clk.step0 + s, wfirst >> 5)] = word;
        }
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) staged_issue_stores<BLOCK, FIXED, IPT>(k, stage, base, W);
    // block-wide delivery: the edges of a chunk's spikers are spread over all its threads (a
    // warp-local delivery leaves one warp with a high out-degree spiker's whole edge list); or,
    // deferred, list entries for the scatter kernel of the step
    if constexpr (DEFER)
      append_spikes<IPT>(k, s, tx_bits, iq, bq, xq);
    else if (!(k.flags & FLYB_LIF_PULL_DELIVERY))
      deliver<BLOCK, FIXED, IPT>(k, sm, tx_bits, iq, bq, xq, ws, slot);
    __syncthreads();
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// Shared memory of the staged kernel, opted in once per instantiation (above the 48 KB default).
template <int BLOCK, bool FIXED, int IPT, bool DEFER>
static int staged_prepare(int* blocks_per_sm) {
  using L = StagedLayout<BLOCK, FIXED, IPT>;
  static int per_sm = -1;
  if (per_sm < 0) {
    cudaError_t e = cudaFuncSetAttribute(lif_staged_kernel<BLOCK, FIXED, IPT, DEFER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
    if (e != cudaSuccess) return (int)e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_staged_kernel<BLOCK, FIXED, IPT, DEFER>, BLOCK,
                                                      L::BYTES);
    if (e != cudaSuccess) return (int)e;
    per_sm = b;
  }
  *blocks_per_sm = per_sm;
  return 0;
}

// The staged path's requirements: 16-byte aligned chunk copies (items of the launch a multiple of
// 4 starting on a multiple of 4, 16-byte aligned arrays).
static bool stageable(const LifK& k) {
  if ((k.t_end - k.t_begin) % 4 || k.t_begin % 4) return false;
  const void* ptrs[] = {k.v, k.g, k.refrac, k.adapt, k.res, k.rate, k.counts, k.spikes, k.drive, k.poisson_p, k.ring};
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) & 15) return false;
  return true;
}

template <int BLOCK, bool FIXED, int IPT, bool DEFER>
static int run_lif_staged_as(const LifK& k, int grid_cap, cudaStream_t st) {
  using L = StagedLayout<BLOCK, FIXED, IPT>;
  if constexpr (L::BYTES > 227 * 1024) return FLYB_EINVAL;   // beyond one block's shared memory
  int per_sm = 0;
  int rc = staged_prepare<BLOCK, FIXED, IPT, DEFER>(&per_sm);
  if (rc) return rc;
  if (per_sm < 1) return FLYB_ECOOP;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long grid = (long long)sms * per_sm;
  const long long chunks = ((long long)k.t_end - k.t_begin + L::CH - 1) / L::CH;
  if (grid > chunks) grid = chunks;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  int pending = 0;
  for (int s = 0; s < k.nsteps; ++s) {
    if constexpr (DEFER) {   // staged update + list, then the balanced scatter
      cudaError_t e = cudaMemsetAsync(k.spike_n, 0, sizeof(unsigned), st);
      if (e != cudaSuccess) return (int)e;
      lif_staged_kernel<BLOCK, FIXED, IPT, true><<<(unsigned)grid, BLOCK, L::BYTES, st>>>(k, s);
      FLYB_CHECK_LAUNCH();
      lif_scatter_kernel<FIXED><<<sms * 8, 256, 0, st>>>(k, s);
    } else {
      lif_staged_kernel<BLOCK, FIXED, IPT><<<(unsigned)grid, BLOCK, L::BYTES, st>>>(k, s);
      FLYB_CHECK_LAUNCH();
      const int rc = pull_after_step(k, s, pending, st);
      if (rc) return rc;
    }
    FLYB_CHECK_LAUNCH();
  }
  if (needs_advance(k)) {
    lif_advance_kernel<<<1, 256, 0, st>>>(k);
    FLYB_CHECK_LAUNCH();
  }
  return 0;
}

template <int BLOCK, bool FIXED, int IPT>
static int run_lif_staged(const LifK& k, int grid_cap, cudaStream_t st) {
  return k.spike_list ? run_lif_staged_as<BLOCK, FIXED, IPT, true>(k, grid_cap, st)
                      : run_lif_staged_as<BLOCK, FIXED, IPT, false>(k, grid_cap, st);
}

template <int BLOCK, bool FIXED, int IPT>
static int run_lif_ipt(const LifK& k, int launch, int grid_cap, cudaStream_t st) {
  const long long W = (long long)k.t_end - k.t_begin;
  const long long chunks = (W + (long long)BLOCK * IPT - 1) / ((long long)BLOCK * IPT);
  if (launch == FLYB_LAUNCH_STEP) {
    int scatter_grid = 0;
    if (k.spike_list) {
      int dev = 0, sms = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      scatter_grid = sms * 8;
    }
    int pending = 0;
    for (int s = 0; s < k.nsteps; ++s) {
      if (k.spike_list) {   // deferred delivery: update + list, then the balanced scatter
        cudaError_t e = cudaMemsetAsync(k.spike_n, 0, sizeof(unsigned), st);
        if (e != cudaSuccess) return (int)e;
        lif_step_kernel<BLOCK, FIXED, IPT, true><<<(unsigned)chunks, BLOCK, 0, st>>>(k, s);
        FLYB_CHECK_LAUNCH();
        lif_scatter_kernel<FIXED><<<scatter_grid, 256, 0, st>>>(k, s);
      } else {
        lif_step_kernel<BLOCK, FIXED, IPT><<<(unsigned)chunks, BLOCK, 0, st>>>(k, s);
        FLYB_CHECK_LAUNCH();
        const int rc = pull_after_step(k, s, pending, st);
        if (rc) return rc;
      }
      FLYB_CHECK_LAUNCH();
    }
    if (needs_advance(k)) {
      lif_advance_kernel<<<1, 256, 0, st>>>(k);
      FLYB_CHECK_LAUNCH();
    }
    return 0;
  }
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lif_persistent_kernel<BLOCK, FIXED, IPT>, BLOCK, 0);
  long long grid = (long long)sms * per_sm;
  if (grid > chunks) grid = chunks;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  if (grid < 1) return FLYB_ECOOP;
  cudaError_t e = cudaMemsetAsync(k.sync, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  LifK kk = k;
  void* args[] = {&kk};
  e = cudaLaunchCooperativeKernel((void*)lif_persistent_kernel<BLOCK, FIXED, IPT>, dim3((unsigned)grid), dim3(BLOCK),
                                  args, 0, st);
  return (int)e;
}

// `ipt` items per thread (8- or 16-byte state vectors) need every ring slot and state array
// aligned at each thread's first item: n * batch % ipt == 0 and (4 * ipt)-byte aligned bases.
static bool vectorizable(const LifK& k, int ipt) {
  if ((k.t_end - k.t_begin) % ipt || k.t_begin % ipt) return false;
  const void* ptrs[] = {k.v, k.g, k.refrac, k.adapt, k.res, k.rate, k.counts, k.spikes, k.drive, k.poisson_p, k.ring};
  for (const void* p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) & (4 * ipt - 1)) return false;
  return true;
}

// Items per thread: the caller's choice when its vectors are aligned, else 4 when possible, else 1.
// `staged` per-step launches take the bulk-copy path when its alignment holds (2 or 4 items per
// thread there: 1 runs as 2).
template <int BLOCK, bool FIXED>
static int run_lif(const LifK& k, int want, int launch, int grid_cap, int staged, cudaStream_t st) {
  int ipt = want ? want : 4;
  if (ipt != 1 && ipt != 2 && ipt != 4) return FLYB_EINVAL;
  if (staged && launch == FLYB_LAUNCH_STEP && stageable(k))
    return ipt == 4 ? run_lif_staged<BLOCK, FIXED, 4>(k, grid_cap, st) : run_lif_staged<BLOCK, FIXED, 2>(k, grid_cap, st);
  while (ipt > 1 && !vectorizable(k, ipt)) ipt >>= 1;
  if (ipt == 4) return run_lif_ipt<BLOCK, FIXED, 4>(k, launch, grid_cap, st);
  if (ipt == 2) return run_lif_ipt<BLOCK, FIXED, 2>(k, launch, grid_cap, st);
  return run_lif_ipt<BLOCK, FIXED, 1>(k, launch, grid_cap, st);
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
  if (block == 128) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<128, false, 4>, 128, 0);
  else if (block == 512) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<512, false, 4>, 512, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lif_persistent_kernel<256, false, 4>, 256, 0);
  return b;
}

}  // namespace flyb

using namespace flyb;

FLYB_API long long flyb_lif_spike_capacity(const flyb_lif_args* a) {
  if (!a || a->n <= 0 || a->batch <= 0 || !a->out_ptr) return -1;
  const int first = a->n_first, count = a->n_count ? a->n_count : a->n - a->n_first;
  if (first < 0 || count <= 0 || (long long)first + count > a->n) return -1;
  // every item of the launch fires: one entry per item plus one per full kEdgeChunk of its edges
  int lo = 0, hi = 0;
  if (cudaMemcpy(&lo, a->out_ptr + first, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&hi, a->out_ptr + first + count, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return (long long)count * a->batch + ((long long)(hi - lo) / kEdgeChunk) * a->batch;
}

// Validates the arguments and fills the kernel view; 0 or an FLYB_E* code.
static int make_lif_k(const flyb_lif_args* a, LifK& k) {
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
  const int count = a->n_count ? a->n_count : a->n - a->n_first;
  if (a->n_first < 0 || a->n_first >= a->n || a->n_count < 0 || count <= 0 || (long long)a->n_first + count > a->n ||
      ((long long)a->n_first * a->batch) % 32)
    return FLYB_EINVAL;
  k.n = a->n; k.batch = a->batch; k.n_delay = a->n_delay; k.R = a->ring_slots; k.flags = a->flags;
  batch_divider(a->batch, &k.bdiv_m, &k.bdiv_s);
  k.t_begin = a->n_first * a->batch;
  k.t_end = (a->n_first + count) * a->batch;
  k.nsteps = a->nsteps; k.ring_pos = ((a->ring_pos % k.R) + k.R) % k.R;
  if (a->raster_slots < 0) return FLYB_EINVAL;
  k.words = (int)(((long long)a->n * a->batch + 31) / 32);
  k.step0 = a->step0; k.seed = a->seed;
  k.out_ptr = a->out_ptr; k.out_edge = (const int2*)a->out_edge;
  k.v = a->v; k.g = a->g; k.refrac = a->refrac; k.adapt = a->adapt; k.res = a->res; k.rate = a->rate;
  k.counts = a->counts; k.spikes = a->spikes; k.drive = a->drive; k.poisson_p = a->poisson_p;
  k.active = a->active; k.std_u = a->std_u; k.ring = a->ring; k.uniforms = a->uniforms; k.fly_steps = a->fly_steps;
  k.clock = a->clock;
  k.raster = a->raster; k.raster_slots = a->raster_slots; k.fly0 = a->fly0;
  k.raster_pos = a->raster_slots > 0 ? ((a->raster_pos % a->raster_slots) + a->raster_slots) % a->raster_slots : 0;
  k.events = a->events; k.status = a->status; k.sync = a->sync;
  k.spike_list = nullptr; k.spike_n = nullptr; k.spike_cap = 0;
  k.adapt_jump = a->adapt_jump;
  k.clock_k = a->clock_k; k.clock_coef = a->clock_coef; k.clock_acc = (long long*)a->clock_acc;
  if (a->clock_k && (!a->clock_coef || !a->clock_acc || (a->flags & FLYB_LIF_DEFER_DELIVERY))) return FLYB_EINVAL;
  k.slow_classes = a->slow_classes; k.slow_mode = a->slow_mode;
  k.slow_norm = a->slow_norm; k.slow_clip_lo = a->slow_clip_lo; k.slow_clip_hi = a->slow_clip_hi;
  k.slow_th_max = a->slow_th_max; k.g_slow = a->g_slow;
  if (a->slow_classes < 0 || a->slow_classes > FLYB_SLOW_MAX_CLASSES) return FLYB_EINVAL;
  if (a->slow_classes) {
    if ((a->flags & FLYB_LIF_DEFER_DELIVERY) || !a->g_slow || a->slow_mode < FLYB_SLOW_ADDITIVE ||
        a->slow_mode > FLYB_SLOW_THRESHOLD || !(a->slow_norm != 0.0f))
      return FLYB_EINVAL;
  }
  for (int c = 0; c < FLYB_SLOW_MAX_CLASSES; ++c) {
    const bool used = c < a->slow_classes;
    if (used && (!a->slow_out_ptr[c] || !a->slow_out_edge[c] || !a->slow_ring[c] || !a->slow_g[c] ||
                 (a->clock_k && !a->slow_clock_acc[c])))
      return FLYB_EINVAL;
    k.slow_clock_acc[c] = used && a->clock_k ? (long long*)a->slow_clock_acc[c] : nullptr;
    k.slow_decay[c] = used ? a->slow_decay[c] : 0.0f;
    k.slow_out_ptr[c] = used ? a->slow_out_ptr[c] : nullptr;
    k.slow_out_edge[c] = used ? (const int2*)a->slow_out_edge[c] : nullptr;
    k.slow_ring[c] = used ? (long long*)a->slow_ring[c] : nullptr;
    k.slow_g[c] = used ? a->slow_g[c] : nullptr;
  }
  k.pull_ptr = a->pull_ptr; k.pull_pre = a->pull_pre; k.pull_planes = a->pull_planes;
  k.pull_nplanes = a->pull_nplanes; k.pull_meta = a->pull_meta;
  k.pull_group = a->pull_group; k.pull_phase = a->pull_phase; k.pull_bits = nullptr; k.pull_state = nullptr;
  k.pull_grid = a->pull_grid;
  if (a->pull_grid < 0) return FLYB_EINVAL;
  k.pull_group_log2 = 0;
  while ((1 << k.pull_group_log2) < a->pull_group && k.pull_group_log2 < 4) ++k.pull_group_log2;
  if (a->flags & FLYB_LIF_PULL_DELIVERY) {
    const int g = a->batch / 32;
    // a group's pull may run beside the next group's updates and must end before the steps after
    // them: its earliest write slot is read n_delay steps after its first step, so 2 L <= n_delay
    if (a->batch % 32 || (g != 1 && g != 2 && g != 4 && g != 8) || a->ring_mode != FLYB_RING_COUNT ||
        a->launch != FLYB_LAUNCH_STEP || (a->flags & (FLYB_LIF_DEFER_DELIVERY | FLYB_LIF_STD)) || a->clock_k ||
        a->slow_classes || !a->pull_ptr || !a->pull_pre || !a->pull_meta ||
        (a->pull_nplanes != 0 && a->pull_nplanes != 16) ||
        (a->pull_nplanes && (!a->pull_planes || (reinterpret_cast<uintptr_t>(a->pull_planes) & 15))) ||
        (a->pull_nplanes == 0 && a->n > (int)kPullPad) ||
        !a->pull_bits || !a->pull_state || (reinterpret_cast<uintptr_t>(a->pull_bits) & 31) ||
        !pull_group_ok(a->batch, a->pull_group) || (a->pull_group > 1 && 2 * a->pull_group > a->n_delay) ||
        a->pull_phase < 0 || a->pull_phase >= a->pull_group)
      return FLYB_EINVAL;
    k.pull_bits = a->pull_bits; k.pull_state = a->pull_state;
  }
  if (a->flags & FLYB_LIF_DEFER_DELIVERY) {
    // per-step launches of the register path only; the list must hold every entry a step can make
    if (!a->spike_list || !a->spike_n || a->spike_cap <= 0 || a->launch != FLYB_LAUNCH_STEP) return FLYB_EINVAL;
    k.spike_list = (int4*)a->spike_list; k.spike_n = a->spike_n; k.spike_cap = a->spike_cap;
  }
  const float* P = a->params;
  k.P = LifP{P[FLYB_P_V_REST], P[FLYB_P_V_RESET], P[FLYB_P_V_TH], P[FLYB_P_A_M], P[FLYB_P_A_S], P[FLYB_P_DT],
             P[FLYB_P_T_REF], P[FLYB_P_ADAPT_JUMP], P[FLYB_P_A_AD], P[FLYB_P_A_STD], P[FLYB_P_A_R],
             P[FLYB_P_RATE_GAIN], P[FLYB_P_W_SYN]};
  return 0;
}

FLYB_API int flyb_lif_advance(const flyb_lif_args* a, void* stream) {
  LifK k;
  const int rc = make_lif_k(a, k);
  if (rc) return rc;
  if (a->nsteps == 0 || !(k.clock || (k.flags & FLYB_LIF_EPISODES))) return 0;
  lif_advance_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(k);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_lif_pull(const flyb_lif_args* a, void* stream) {
  LifK k;
  const int rc = make_lif_k(a, k);
  if (rc) return rc;
  if (!(k.flags & FLYB_LIF_PULL_DELIVERY) || a->pull_steps < 1 || a->pull_steps > k.pull_group) return FLYB_EINVAL;
  return launch_pull(k, a->pull_steps, (cudaStream_t)stream);
}

FLYB_API int flyb_lif_run(const flyb_lif_args* a, void* stream) {
  LifK k;
  const int rc = make_lif_k(a, k);
  if (rc) return rc;
  if (a->nsteps == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  const bool fixed = a->ring_mode == FLYB_RING_FIXED;
  const int block = a->block ? a->block : 256;
  if (k.clock_k || k.slow_classes) {
    if (block != 128 && block != 256 && block != 512) return FLYB_EINVAL;
    return fixed ? run_lif_ext<256, true>(k, st) : run_lif_ext<256, false>(k, st);
  }
  switch (block) {
    case 128: return fixed ? run_lif<128, true>(k, a->items_per_thread, a->launch, a->grid, a->staged, st)
                     : run_lif<128, false>(k, a->items_per_thread, a->launch, a->grid, a->staged, st);
    case 256: return fixed ? run_lif<256, true>(k, a->items_per_thread, a->launch, a->grid, a->staged, st)
                     : run_lif<256, false>(k, a->items_per_thread, a->launch, a->grid, a->staged, st);
    case 512: return fixed ? run_lif<512, true>(k, a->items_per_thread, a->launch, a->grid, a->staged, st)
                     : run_lif<512, false>(k, a->items_per_thread, a->launch, a->grid, a->staged, st);
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
