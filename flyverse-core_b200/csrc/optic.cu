// Optic-lobe rate step for sm_100a: CSR SpMV/SpMM y = W_rr @ dr fused with the rate update
// (flyverse/optic.py:_substep, optic.py:525-551; neural.cu:62-88), the held-input products
// (optic.py:579-580, 599-602) and the reference-compatible elementwise / CSR launchers.
//
// Layout: state [m][batch] (unit-major, fly-minor); CSR entries interleaved as int2 {col, w bits}.
// A warp holds 32/LPR row slots; in a slot F lanes span the flies (FPL consecutive flies each: a
// 4-, 8- or 16-byte vector gather of x[col][*]) and LPR/F lane groups split the entries, each lane
// keeping U independent gathers in flight. Rows run longest first; rows longer than a threshold
// are split over every slot of a block and summed through shared memory. The gathered vector
// (dr, 0.36 MB per fly) stays L2-resident; the CSR streams from HBM once per substep for all flies.
// Substeps ping-pong dr between two buffers, so one grid barrier per substep suffices, and the dr
// of the final state is left for the next call (FLYB_OPTIC_DR_VALID).
#include <mutex>

#include "common.cuh"

namespace flyb {

struct OpticK {
  int m, batch, nsteps;
  const int* __restrict__ ptr; const int2* __restrict__ cw;
  const int* __restrict__ rows;   // optional row order: rows[0, n_long) long rows, then the others
  int n_long;
  float* __restrict__ v; float* __restrict__ adapt;
  float* buf0; float* buf1;
  const float* __restrict__ pr; const float* __restrict__ spk;
  const float* __restrict__ a; const float* __restrict__ b;
  float gr, ga, aad;
  float* v_hist; float* inp_hist;
  int* status; int* sync;
  int dr_valid;                   // buf0 already holds clip(v + b) - b: no initialisation pass
};

template <int FPL> struct VecT;
template <> struct VecT<1> { using T = float; };
template <> struct VecT<2> { using T = float2; };
template <> struct VecT<4> { using T = float4; };

template <int FPL>
__device__ __forceinline__ void load_x(const float* __restrict__ p, float (&x)[FPL]) {
  if constexpr (FPL == 1) {
    x[0] = __ldg(p);
  } else if constexpr (FPL == 2) {
    const float2 q = __ldg(reinterpret_cast<const float2*>(p)); x[0] = q.x; x[1] = q.y;
  } else if constexpr (FPL == 4) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p)); x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
  } else {
#pragma unroll
    for (int q = 0; q < FPL; q += 4) {
      const float4 r = __ldg(reinterpret_cast<const float4*>(p + q));
      x[q] = r.x; x[q + 1] = r.y; x[q + 2] = r.z; x[q + 3] = r.w;
    }
  }
}

// Entries each lane keeps in flight: the gathers are L2 round trips, so a warp must issue many
// independent ones before it consumes any (fewer when each gather is already a wide vector).
template <int FPL>
struct Unroll { static constexpr int U = FPL <= 2 ? 8 : (FPL == 4 ? 4 : 2); };

// acc[q] = sum over the row of w * x[col][f*FPL + q] for this lane's flies, for the row of this
// lane's slot: a warp holds 32/LPR row slots of LPR lanes; within a slot, F lanes span the flies
// (FPL consecutive flies each) and G = LPR/F lane groups split the entries (group g takes entries
// e0 + g + G*k). Each pass loads U interleaved {col, w} entries (8 bytes each), issues U
// independent gathers, then accumulates them with FMAs. The result is complete on the lanes with
// slot lane < F. `row_ok` false: the lane still takes part in the shuffles.
template <int F, int FPL, int LPR, int U = Unroll<FPL>::U>
__device__ __forceinline__ void row_product(const int* __restrict__ ptr, const int2* __restrict__ cw,
                                            const float* __restrict__ x, int batch, int row, bool row_ok,
                                            float (&acc)[FPL], int part = 0, int parts = 1) {
  static_assert(F <= LPR && LPR <= 32, "a row slot spans the fly lanes");
  constexpr int G = LPR / F;
  const int sl = (threadIdx.x & 31) % LPR, g = sl / F, f = sl % F;
  const int fb = f * FPL;
  const bool full = batch == F * FPL;
  const int stride = parts * G;          // `parts` slots share a long row: slot `part` takes every parts-th group
#pragma unroll
  for (int q = 0; q < FPL; ++q) acc[q] = 0.0f;
  if (row_ok) {
    const int e0 = __ldg(&ptr[row]), e1 = __ldg(&ptr[row + 1]);
    for (int base = e0 + part * G + g; base < e1; base += stride * U) {
      int2 c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = base + u * stride;
        c[u] = e < e1 ? __ldg(&cw[e]) : make_int2(-1, 0);
      }
      float xv[U][FPL];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const float* xp = x + ((c[u].x < 0 ? 0 : c[u].x) * batch + fb);
        if (full) {
          load_x<FPL>(xp, xv[u]);
        } else {
#pragma unroll
          for (int q = 0; q < FPL; ++q) xv[u][q] = fb + q < batch ? __ldg(xp + q) : 0.0f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (c[u].x >= 0) {
          const float wv = __int_as_float(c[u].y);
#pragma unroll
          for (int q = 0; q < FPL; ++q) acc[q] = fmaf(wv, xv[u][q], acc[q]);
        }
      }
    }
  }
#pragma unroll
  for (int o = F; o < LPR; o <<= 1)
#pragma unroll
    for (int q = 0; q < FPL; ++q) acc[q] = acc[q] + __shfl_xor_sync(0xffffffffu, acc[q], o);
}

// The fused rate update of one (unit, fly), reference order (neural.cu:68-79, optic.py:528-551).
__device__ __forceinline__ void optic_update(const OpticK& k, int s, size_t t, int i, float y,
                                             const float* __restrict__ dr_in, float* __restrict__ dr_out) {
  const float old = dr_in[t];
  float inp = k.gr * y;
  inp = inp + k.pr[t];
  const float ad = k.ga * k.adapt[t];
  inp = inp - ad;
  inp = inp + k.spk[t];
  float vv = k.v[t];
  const size_t sz = (size_t)k.m * k.batch;
  if (k.v_hist) k.v_hist[(size_t)s * sz + t] = vv;
  if (k.inp_hist) k.inp_hist[(size_t)s * sz + t] = inp;
  float dv = vv - inp;
  dv = dv * k.a[i];
  vv = inp + dv;
  k.v[t] = vv;
  float da = k.adapt[t] - old;
  da = da * k.aad;
  k.adapt[t] = old + da;
  const float bb = k.b[i];
  const float r = clip01(vv + bb);
  dr_out[t] = r - bb;
}

template <int FPL>
__device__ __forceinline__ void store_x(float* p, const float (&x)[FPL]) {
  if constexpr (FPL == 1) {
    *p = x[0];
  } else if constexpr (FPL == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(x[0], x[1]);
  } else {
#pragma unroll
    for (int q = 0; q < FPL; q += 4) *reinterpret_cast<float4*>(p + q) = make_float4(x[q], x[q + 1], x[q + 2], x[q + 3]);
  }
}

// The same update for FPL consecutive flies of one unit with vector loads and stores (batch == F*FPL).
template <int FPL>
__device__ __forceinline__ void optic_update_vec(const OpticK& k, int s, size_t t, int i, const float (&y)[FPL],
                                                 const float* __restrict__ dr_in, float* __restrict__ dr_out) {
  float old[FPL], pr[FPL], spk[FPL], ad[FPL], vv[FPL];
  load_x<FPL>(dr_in + t, old);
  load_x<FPL>(k.pr + t, pr);
  load_x<FPL>(k.spk + t, spk);
  load_x<FPL>(k.adapt + t, ad);
  load_x<FPL>(k.v + t, vv);
  const float ai = k.a[i], bb = k.b[i];
  const size_t sz = (size_t)k.m * k.batch;
  if (k.v_hist) store_x<FPL>(k.v_hist + (size_t)s * sz + t, vv);
  float inpv[FPL], nv[FPL], na[FPL], nd[FPL];
#pragma unroll
  for (int q = 0; q < FPL; ++q) {
    float inp = k.gr * y[q];
    inp = inp + pr[q];
    const float a2 = k.ga * ad[q];
    inp = inp - a2;
    inp = inp + spk[q];
    inpv[q] = inp;
    float dv = vv[q] - inp;
    dv = dv * ai;
    nv[q] = inp + dv;
    float da = ad[q] - old[q];
    da = da * k.aad;
    na[q] = old[q] + da;
    nd[q] = clip01(nv[q] + bb) - bb;
  }
  if (k.inp_hist) store_x<FPL>(k.inp_hist + (size_t)s * sz + t, inpv);
  store_x<FPL>(k.v + t, nv);
  store_x<FPL>(k.adapt + t, na);
  store_x<FPL>(dr_out + t, nd);
}

// y (FPL flies of slot lane sl) -> the fused update of one unit.
template <int F, int FPL>
__device__ __forceinline__ void optic_epilogue(const OpticK& k, int s, int row, int sl, const float (&y)[FPL],
                                               const float* dr_in, float* dr_out) {
  if (k.batch == F * FPL) {
    optic_update_vec<FPL>(k, s, (size_t)row * k.batch + sl * FPL, row, y, dr_in, dr_out);
  } else {
#pragma unroll
    for (int q = 0; q < FPL; ++q) {
      const int bb = sl * FPL + q;
      if (bb < k.batch) optic_update(k, s, (size_t)row * k.batch + bb, row, y[q], dr_in, dr_out);
    }
  }
}

template <int F, int FPL, int LPR>
struct OpticShape {
  static constexpr int RPW = 32 / LPR;           // row slots per warp
  static constexpr int SLOTS = 8 * RPW;          // row slots per 256-thread block
  static constexpr int RED = SLOTS * F * FPL;    // floats of the long-row reduction
};

// Number of block work items of one substep: one per long row, then blocks of SLOTS short rows.
template <int F, int FPL, int LPR>
__host__ __device__ __forceinline__ long long optic_items(int m, int n_long) {
  constexpr int SLOTS = OpticShape<F, FPL, LPR>::SLOTS;
  return n_long + (m - n_long + SLOTS - 1) / SLOTS;
}

// One block work item. Long rows (the first n_long of k.rows): every row slot of the block takes an
// interleaved share of the row's entries, the shares are summed in slot order through shared
// memory and the first slot applies the update; the longest rows thus stop bounding the substep.
// Other rows: one row per slot.
template <int F, int FPL, int LPR, int U>
__device__ __forceinline__ void optic_item(const OpticK& k, int s, const float* dr_in, float* dr_out, long long item,
                                           float* red) {
  using S = OpticShape<F, FPL, LPR>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, slot = lane / LPR, sl = lane % LPR;
  const int gslot = warp * S::RPW + slot;
  float acc[FPL];
  if (item < k.n_long) {
    const int row = k.rows[item];
    row_product<F, FPL, LPR, U>(k.ptr, k.cw, dr_in, k.batch, row, true, acc, gslot, S::SLOTS);
    if (sl < F) {
#pragma unroll
      for (int q = 0; q < FPL; ++q) red[gslot * F * FPL + sl * FPL + q] = acc[q];
    }
    __syncthreads();
    if (gslot == 0 && sl < F) {
      float y[FPL];
#pragma unroll
      for (int q = 0; q < FPL; ++q) y[q] = red[sl * FPL + q];
      for (int p = 1; p < S::SLOTS; ++p)
#pragma unroll
        for (int q = 0; q < FPL; ++q) y[q] = y[q] + red[p * F * FPL + sl * FPL + q];
      optic_epilogue<F, FPL>(k, s, row, sl, y, dr_in, dr_out);
    }
    __syncthreads();
  } else {
    const long long r = k.n_long + (item - k.n_long) * S::SLOTS + gslot;
    const bool ok = r < k.m;
    const int row = ok ? (k.rows ? k.rows[r] : (int)r) : 0;
    row_product<F, FPL, LPR, U>(k.ptr, k.cw, dr_in, k.batch, row, ok, acc);
    if (ok && sl < F) optic_epilogue<F, FPL>(k, s, row, sl, acc, dr_in, dr_out);
  }
}

// dr = clip(v + b, 0, 1) - b over the state (m * batch < 2^31, checked by the entry points).
__device__ __forceinline__ void init_dr(const OpticK& k, float* dr, int tid, int nthreads) {
  const int sz = k.m * k.batch;
  for (int t = tid; t < sz; t += nthreads) {
    const float bb = __ldg(&k.b[t / k.batch]);
    dr[t] = clip01(k.v[t] + bb) - bb;
  }
}

__global__ void optic_init_kernel(OpticK k) {
  init_dr(k, k.buf0, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// MINB: blocks per SM the registers must allow (launch bounds); 8 caps them at 32 per thread so a
// full SM of 64 warps keeps gathers in flight.
template <int F, int FPL, int LPR, int U, int MINB>
__global__ void __launch_bounds__(256, MINB) optic_step_kernel(OpticK k, int s) {
  __shared__ float red[OpticShape<F, FPL, LPR>::RED];
  const float* in = (s & 1) ? k.buf1 : k.buf0;
  float* out = (s & 1) ? k.buf0 : k.buf1;
  optic_item<F, FPL, LPR, U>(k, s, in, out, blockIdx.x, red);
}

template <int F, int FPL, int LPR, int U, int MINB>
__global__ void __launch_bounds__(256, MINB) optic_persistent_kernel(OpticK k) {
  __shared__ float red[OpticShape<F, FPL, LPR>::RED];
  int generation = 0;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  const long long items = optic_items<F, FPL, LPR>(k.m, k.n_long);
  if (!k.dr_valid) {
    init_dr(k, k.buf0, (int)tid, (int)nth);
    if (!grid_barrier(k.sync, k.status, generation, -1)) return;
  }
  for (int s = 0; s < k.nsteps; ++s) {
    const float* in = (s & 1) ? k.buf1 : k.buf0;
    float* out = (s & 1) ? k.buf0 : k.buf1;
    for (long long item = blockIdx.x; item < items; item += gridDim.x) optic_item<F, FPL, LPR, U>(k, s, in, out, item, red);
    if (s + 1 < k.nsteps && !grid_barrier(k.sync, k.status, generation, s)) return;
  }
}

template <int F, int FPL, int LPR, int U = Unroll<FPL>::U, int MINB = 1>
static int run_optic(const OpticK& k, int launch, int grid_cap, cudaStream_t st) {
  const long long sz = (long long)k.m * k.batch;
  if (launch == FLYB_LAUNCH_STEP) {
    if (!k.dr_valid) {
      optic_init_kernel<<<(unsigned)((sz + 255) / 256), 256, 0, st>>>(k);
      FLYB_CHECK_LAUNCH();
    }
    const unsigned blocks = (unsigned)optic_items<F, FPL, LPR>(k.m, k.n_long);
    for (int s = 0; s < k.nsteps; ++s) {
      optic_step_kernel<F, FPL, LPR, U, MINB><<<blocks, 256, 0, st>>>(k, s);
      FLYB_CHECK_LAUNCH();
    }
    return 0;
  }
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, optic_persistent_kernel<F, FPL, LPR, U, MINB>, 256, 0);
  long long grid = (long long)sms * per_sm;
  const long long need = optic_items<F, FPL, LPR>(k.m, k.n_long);
  if (grid > need) grid = need;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  if (grid < 1) return FLYB_ECOOP;
  if (k.nsteps == 1 && k.dr_valid) {
    // one substep on a carried dr reaches no grid barrier: an ordinary launch of `grid` blocks
    // looping over the items, which other kernels may share the SMs with
    optic_persistent_kernel<F, FPL, LPR, U, MINB><<<(unsigned)grid, 256, 0, st>>>(k);
    return (int)cudaGetLastError();
  }
  cudaError_t e = cudaMemsetAsync(k.sync, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  OpticK kk = k;
  void* args[] = {&kk};
  e = cudaLaunchCooperativeKernel((void*)optic_persistent_kernel<F, FPL, LPR, U, MINB>, dim3((unsigned)grid), dim3(256), args, 0,
                                  st);
  return (int)e;
}

// Picks (F, FPL) from the batch: F lanes across flies, FPL consecutive flies per lane.
#define FLYB_BATCH_DISPATCH(B, CALL)                                   \
  do {                                                                 \
    if ((B) == 1) { constexpr int F = 1, FPL = 1; return CALL; }       \
    if ((B) <= 2) { constexpr int F = 2, FPL = 1; return CALL; }       \
    if ((B) <= 4) { constexpr int F = 4, FPL = 1; return CALL; }       \
    if ((B) <= 8) { constexpr int F = 8, FPL = 1; return CALL; }       \
    if ((B) <= 16) { constexpr int F = 16, FPL = 1; return CALL; }     \
    if ((B) <= 32) { constexpr int F = 32, FPL = 1; return CALL; }     \
    if ((B) <= 64) { constexpr int F = 32, FPL = 2; return CALL; }     \
    if ((B) <= 128) { constexpr int F = 32, FPL = 4; return CALL; }    \
    if ((B) <= 256) { constexpr int F = 32, FPL = 8; return CALL; }    \
    return FLYB_ETOOBIG;                                               \
  } while (0)

// (F fly lanes, FPL flies per lane) of the held-input products: from 32 flies on, 4 flies per lane
// so that a warp instruction covers 2-4 entries (the per-entry index and weight work is shared by
// more products).
#define FLYB_SPMM_DISPATCH(B, CALL)                                    \
  do {                                                                 \
    if ((B) == 1) { constexpr int F = 1, FPL = 1; return CALL; }       \
    if ((B) <= 2) { constexpr int F = 2, FPL = 1; return CALL; }       \
    if ((B) <= 4) { constexpr int F = 4, FPL = 1; return CALL; }       \
    if ((B) <= 8) { constexpr int F = 8, FPL = 1; return CALL; }       \
    if ((B) <= 16) { constexpr int F = 16, FPL = 1; return CALL; }     \
    if ((B) <= 32) { constexpr int F = 8, FPL = 4; return CALL; }      \
    if ((B) <= 64) { constexpr int F = 16, FPL = 4; return CALL; }     \
    if ((B) <= 128) { constexpr int F = 32, FPL = 4; return CALL; }    \
    if ((B) <= 256) { constexpr int F = 32, FPL = 8; return CALL; }    \
    return FLYB_ETOOBIG;                                               \
  } while (0)

// (F fly lanes, FPL flies per lane, LPR lanes per row, U gathers in flight per lane, MINB blocks per
// SM) of the optic substep for a batch; `variant` 0 is the default, the others are alternatives the
// autotuner tries (more warps with fewer registers each, or wider lanes); an unknown variant is an
// error.
#define FLYB_OPTIC_DISPATCH(B, V, CALL)                                                           \
  do {                                                                                            \
    if ((B) == 1) {                                                                               \
      if ((V) == 0) { constexpr int F = 1, FPL = 1, LPR = 8, U = 8, MINB = 1; return CALL; }      \
      if ((V) == 1) { constexpr int F = 1, FPL = 1, LPR = 16, U = 8, MINB = 1; return CALL; }     \
      if ((V) == 2) { constexpr int F = 1, FPL = 1, LPR = 32, U = 8, MINB = 1; return CALL; }     \
      if ((V) == 3) { constexpr int F = 1, FPL = 1, LPR = 8, U = 4, MINB = 8; return CALL; }      \
      if ((V) == 4) { constexpr int F = 1, FPL = 1, LPR = 16, U = 4, MINB = 8; return CALL; }     \
      return FLYB_EINVAL;                                                                         \
    }                                                                                             \
    if ((V) != 0 && (B) <= 32) return FLYB_EINVAL;                                                \
    if ((B) <= 2) { constexpr int F = 2, FPL = 1, LPR = 16, U = 8, MINB = 1; return CALL; }       \
    if ((B) <= 4) { constexpr int F = 4, FPL = 1, LPR = 16, U = 8, MINB = 1; return CALL; }       \
    if ((B) <= 8) { constexpr int F = 8, FPL = 1, LPR = 32, U = 8, MINB = 1; return CALL; }       \
    if ((B) <= 16) { constexpr int F = 16, FPL = 1, LPR = 32, U = 8, MINB = 1; return CALL; }     \
    if ((B) <= 32) { constexpr int F = 32, FPL = 1, LPR = 32, U = 8, MINB = 1; return CALL; }     \
    if ((B) <= 64) {                                                                              \
      if ((V) == 0) { constexpr int F = 16, FPL = 4, LPR = 32, U = 4, MINB = 1; return CALL; }    \
      if ((V) == 1) { constexpr int F = 32, FPL = 2, LPR = 32, U = 8, MINB = 1; return CALL; }    \
      if ((V) == 2) { constexpr int F = 8, FPL = 8, LPR = 32, U = 2, MINB = 1; return CALL; }     \
      if ((V) == 3) { constexpr int F = 16, FPL = 4, LPR = 32, U = 2, MINB = 8; return CALL; }    \
      if ((V) == 4) { constexpr int F = 32, FPL = 2, LPR = 32, U = 4, MINB = 8; return CALL; }    \
      if ((V) == 5) { constexpr int F = 16, FPL = 4, LPR = 32, U = 4, MINB = 6; return CALL; }    \
      return FLYB_EINVAL;                                                                         \
    }                                                                                             \
    if ((B) <= 128) {                                                                             \
      if ((V) == 0) { constexpr int F = 32, FPL = 4, LPR = 32, U = 4, MINB = 1; return CALL; }    \
      if ((V) == 1) { constexpr int F = 16, FPL = 8, LPR = 32, U = 2, MINB = 1; return CALL; }    \
      if ((V) == 3) { constexpr int F = 32, FPL = 4, LPR = 32, U = 2, MINB = 8; return CALL; }    \
      return FLYB_EINVAL;                                                                         \
    }                                                                                             \
    if ((B) <= 256) {                                                                             \
      if ((V) == 0) { constexpr int F = 32, FPL = 8, LPR = 32, U = 2, MINB = 1; return CALL; }    \
      if ((V) == 1) { constexpr int F = 32, FPL = 8, LPR = 32, U = 2, MINB = 4; return CALL; }    \
      if ((V) == 3) { constexpr int F = 32, FPL = 8, LPR = 32, U = 1, MINB = 6; return CALL; }    \
      if ((V) == 5) { constexpr int F = 32, FPL = 8, LPR = 32, U = 1, MINB = 8; return CALL; }    \
      return FLYB_EINVAL;                                                                         \
    }                                                                                             \
    return FLYB_ETOOBIG;                                                                          \
  } while (0)

// ------------------------------------------------------------------ held-input products
struct SpmmK {
  int rows, batch, accumulate;
  const int* __restrict__ ptr; const int* __restrict__ col; const float* __restrict__ w;
  const float* __restrict__ x; const int* __restrict__ x_index;
  float x_div, x_lo, x_hi;
  float* y; const int* __restrict__ y_index;
  float alpha, y_lo, y_hi;
  int xvec;   // batch == F * FPL and x aligned to FPL floats: one vector gather per entry and lane
};

// WPR warps share one row (RB = 8 / WPR rows per 256-thread block): warp `part` of a row takes the
// entry groups part, part + WPR, ... of it, the partial sums meet in shared memory and the row's
// first warp applies alpha, the clamp and the store. Lanes: F across the flies (FPL each), G = 32/F
// entry groups per warp.
// XT: the input has a transform (x / x_div clamped to [x_lo, x_hi]); without one the products are
// plain w * x.
template <int F, int FPL, int WPR, bool XT>
__global__ void __launch_bounds__(256) spmm_kernel(SpmmK k) {
  constexpr int G = 32 / F, RB = 8 / WPR;
  constexpr int U = Unroll<FPL>::U;
  __shared__ float red[WPR > 1 ? 8 * F * FPL : 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane / F, f = lane % F, fb = f * FPL;
  const int part = warp % WPR;
  const long long row = (long long)blockIdx.x * RB + warp / WPR;
  const bool ok = row < k.rows;
  float acc[FPL];
#pragma unroll
  for (int q = 0; q < FPL; ++q) acc[q] = 0.0f;
  if (ok) {
    const int e0 = k.ptr[row], e1 = k.ptr[row + 1];
    constexpr int stride = WPR * G;
    for (int base = e0 + part * G + g; base < e1; base += stride * U) {
      int jj[U];
      float ww[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = base + u * stride;
        const bool in = e < e1;
        int j = in ? __ldg(&k.col[e]) : -1;
        if (in && k.x_index) j = __ldg(&k.x_index[j]);
        jj[u] = j;
        ww[u] = in ? __ldg(&k.w[e]) : 0.0f;
      }
      float xv[U][FPL];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k.xvec) {
          load_x<FPL>(k.x + (size_t)(jj[u] < 0 ? 0 : jj[u]) * k.batch + fb, xv[u]);
        } else {
#pragma unroll
          for (int q = 0; q < FPL; ++q)
            xv[u][q] = (jj[u] >= 0 && fb + q < k.batch) ? __ldg(&k.x[(size_t)jj[u] * k.batch + fb + q]) : 0.0f;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0) {
#pragma unroll
          for (int q = 0; q < FPL; ++q) {
            float x = xv[u][q];
            if (XT) {
              if (k.x_div != 1.0f) x = x / k.x_div;   // x / 1 == x exactly: skip the IEEE division
              x = x < k.x_lo ? k.x_lo : (x > k.x_hi ? k.x_hi : x);
            }
            const float p = ww[u] * x;
            acc[q] = acc[q] + p;
          }
        }
      }
    }
  }
#pragma unroll
  for (int o = F; o < 32; o <<= 1)
#pragma unroll
    for (int q = 0; q < FPL; ++q) acc[q] = acc[q] + __shfl_xor_sync(0xffffffffu, acc[q], o);
  if (WPR > 1) {
    if (lane < F)
#pragma unroll
      for (int q = 0; q < FPL; ++q) red[(warp * F + f) * FPL + q] = acc[q];
    __syncthreads();
    if (part == 0 && lane < F)
      for (int p = 1; p < WPR; ++p)
#pragma unroll
        for (int q = 0; q < FPL; ++q) acc[q] = acc[q] + red[((warp + p) * F + f) * FPL + q];
  }
  if (ok && part == 0 && lane < F) {
    const long long yi = k.y_index ? k.y_index[row] : row;
#pragma unroll
    for (int q = 0; q < FPL; ++q) {
      const int bb = fb + q;
      if (bb < k.batch) {
        float r = k.alpha * acc[q];
        r = r < k.y_lo ? k.y_lo : (r > k.y_hi ? k.y_hi : r);
        float* yp = k.y + (size_t)yi * k.batch + bb;
        *yp = k.accumulate ? *yp + r : r;
      }
    }
  }
}

template <int F, int FPL, bool XT>
static int run_spmm_xt(const SpmmK& k, int wpr, unsigned blocks, cudaStream_t st) {
  switch (wpr) {
    case 1: spmm_kernel<F, FPL, 1, XT><<<blocks, 256, 0, st>>>(k); break;
    case 2: spmm_kernel<F, FPL, 2, XT><<<blocks, 256, 0, st>>>(k); break;
    case 4: spmm_kernel<F, FPL, 4, XT><<<blocks, 256, 0, st>>>(k); break;
    case 8: spmm_kernel<F, FPL, 8, XT><<<blocks, 256, 0, st>>>(k); break;
    default: return FLYB_EINVAL;
  }
  return (int)cudaGetLastError();
}

template <int F, int FPL>
static int run_spmm(const SpmmK& k0, int wpr, cudaStream_t st) {
  SpmmK k = k0;
  k.xvec = k.batch == F * FPL && (reinterpret_cast<uintptr_t>(k.x) % (FPL * sizeof(float))) == 0;
  const long long rb = 8 / wpr;
  const unsigned blocks = (unsigned)((k.rows + rb - 1) / rb);
  if (!blocks) return 0;
  const bool xt = k.x_div != 1.0f || k.x_lo > -INFINITY || k.x_hi < INFINITY;
  return xt ? run_spmm_xt<F, FPL, true>(k, wpr, blocks, st) : run_spmm_xt<F, FPL, false>(k, wpr, blocks, st);
}

// ------------------------------------------------------------------ reference-compatible launchers
__global__ void ref_optic_dr_kernel(const float* v, const float* b, float* dr, int n, long long total) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total) { const float base = b[t % n]; dr[t] = clip01(v[t] + base) - base; }
}

struct RefOptic { float *v, *adapt, *dr, *y, *pr, *spk, *a, *b; };

__global__ void ref_optic_kernel(RefOptic s, int n, long long total, float gr, float ga, float aad) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int i = (int)(t % n);
  const float old = s.dr[t];
  float inp = gr * s.y[t];
  inp = inp + s.pr[t];
  const float ad = ga * s.adapt[t];
  inp = inp - ad;
  inp = inp + s.spk[t];
  float dv = s.v[t] - inp;
  dv = dv * s.a[i];
  const float v = inp + dv;
  s.v[t] = v;
  float da = s.adapt[t] - old;
  da = da * aad;
  s.adapt[t] = old + da;
  s.dr[t] = clip01(v + s.b[i]) - s.b[i];
}

// Warp per (fly, row) with a fixed shuffle tree, batch-major (neural.cu:90-104).
template <typename W>
__global__ void ref_csr_kernel(const int* __restrict__ ptr, const int* __restrict__ idx, const W* __restrict__ w,
                               const float* __restrict__ x, float* out, int rows, int cols, int batch) {
  const int lane = threadIdx.x & 31;
  const long long gid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gid >= (long long)rows * batch) return;
  const int b = (int)(gid / rows), row = (int)(gid - (long long)b * rows);
  float sum = 0.0f;
  for (int e = ptr[row] + lane; e < ptr[row + 1]; e += 32) {
    float xv = x[(size_t)b * cols + idx[e]];
    if (sizeof(W) == 2) xv = __half2float(__float2half_rn(xv));
    const float p = (float)w[e] * xv;
    sum = sum + p;
  }
#pragma unroll
  for (int k = 16; k; k >>= 1) sum = sum + __shfl_down_sync(0xffffffffu, sum, k);
  if (lane == 0) out[gid] = sum;
}

int optic_blocks_per_sm() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, optic_persistent_kernel<1, 1, 8, 8, 1>, 256, 0);
  return b;
}

}  // namespace flyb

using namespace flyb;

FLYB_API int flyb_optic_run(const flyb_optic_args* a, void* stream) {
  if (!a || a->m <= 0 || a->batch <= 0 || a->nsteps < 0 || !a->ptr || !a->v || !a->adapt ||
      !a->dr || !a->dr_tmp || !a->pr || !a->spk || !a->a || !a->b)
    return FLYB_EINVAL;
  if ((long long)a->m * a->batch >= (1ll << 31)) return FLYB_ETOOBIG;
  if (a->launch == FLYB_LAUNCH_PERSISTENT && (!a->sync || !a->status)) return FLYB_EINVAL;
  if (a->nsteps == 0) return 0;
  if (a->n_long < 0 || a->n_long > a->m || (a->n_long && !a->rows)) return FLYB_EINVAL;
  OpticK k{a->m, a->batch, a->nsteps, a->ptr, (const int2*)a->cw, a->rows, a->n_long, a->v, a->adapt, a->dr, a->dr_tmp,
           a->pr, a->spk,
           a->a, a->b, a->gr, a->ga, a->aad, (a->flags & FLYB_OPTIC_HISTORY) ? a->v_hist : nullptr,
           (a->flags & FLYB_OPTIC_HISTORY) ? a->inp_hist : nullptr, a->status, a->sync,
           (a->flags & FLYB_OPTIC_DR_VALID) ? 1 : 0};
  cudaStream_t st = (cudaStream_t)stream;
  FLYB_OPTIC_DISPATCH(a->batch, a->variant, (run_optic<F, FPL, LPR, U, MINB>(k, a->launch, a->grid, st)));
}

// ------------------------------------------------------------------ allocation-free variant
// Scratch of flyb_optic_run_noalloc: the two dr ping-pong buffers (FLYB_OPTIC_NOALLOC_MAX floats
// each) and the grid-barrier words, in one file-scope device array. Every GPU that loads this
// library holds it (8 MiB + 256 B) until the process exits.
static __device__ __align__(256) float g_optic_scratch[2 * FLYB_OPTIC_NOALLOC_MAX + 64];

// Device address of g_optic_scratch per device ordinal. Host code must not hand the symbol itself
// to a kernel (on the host it is a stand-in, not a device address): the address is looked up once
// per device, with that device current, by cudaGetSymbolAddress.
static std::mutex g_scratch_mu;
static float* g_scratch_addr[256];

static int optic_noalloc_scratch(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 256) return FLYB_EINVAL;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_optic_scratch);
    if (e != cudaSuccess || !p) return e != cudaSuccess ? (int)e : FLYB_EINVAL;
    g_scratch_addr[dev] = (float*)p;
  }
  *out = g_scratch_addr[dev];
  return 0;
}

FLYB_API int flyb_optic_run_noalloc(const flyb_optic_args* a, void* stream) {
  if (!a || a->m <= 0 || a->batch <= 0 || a->nsteps < 0 || !a->ptr || !a->v || !a->adapt || !a->pr || !a->spk ||
      !a->a || !a->b)
    return FLYB_EINVAL;
  if ((long long)a->m * a->batch > FLYB_OPTIC_NOALLOC_MAX) return FLYB_ETOOBIG;
  if (a->launch == FLYB_LAUNCH_PERSISTENT && !a->status) return FLYB_EINVAL;
  float* scratch = nullptr;
  const int rc = optic_noalloc_scratch(&scratch);
  if (rc) return rc;
  if (a->nsteps == 0) return 0;
  if (a->n_long < 0 || a->n_long > a->m || (a->n_long && !a->rows)) return FLYB_EINVAL;
  OpticK k{a->m, a->batch, a->nsteps, a->ptr, (const int2*)a->cw, a->rows, a->n_long, a->v, a->adapt, scratch,
           scratch + FLYB_OPTIC_NOALLOC_MAX,
           a->pr, a->spk, a->a, a->b, a->gr, a->ga, a->aad, (a->flags & FLYB_OPTIC_HISTORY) ? a->v_hist : nullptr,
           (a->flags & FLYB_OPTIC_HISTORY) ? a->inp_hist : nullptr, a->status,
           (int*)(scratch + 2 * FLYB_OPTIC_NOALLOC_MAX), 0};
  cudaStream_t st = (cudaStream_t)stream;
  FLYB_OPTIC_DISPATCH(a->batch, a->variant, (run_optic<F, FPL, LPR, U, MINB>(k, a->launch, a->grid, st)));
}

FLYB_API int flyb_spmm(const flyb_spmm_args* a, void* stream) {
  if (!a || a->rows < 0 || a->batch <= 0 || !a->ptr || !a->x || !a->y || a->x_div == 0.0f)
    return FLYB_EINVAL;
  if (a->rows == 0) return 0;
  SpmmK k{a->rows, a->batch, a->accumulate, a->ptr, a->col, a->w, a->x, a->x_index, a->x_div, a->x_lo, a->x_hi,
          a->y, a->y_index, a->alpha, a->y_lo, a->y_hi, 0};
  cudaStream_t st = (cudaStream_t)stream;
  const int wpr = a->warps_per_row ? a->warps_per_row : 1;
  if (wpr != 1 && wpr != 2 && wpr != 4 && wpr != 8) return FLYB_EINVAL;
  FLYB_SPMM_DISPATCH(a->batch, (run_spmm<F, FPL>(k, wpr, st)));
}

FLYB_API int launch_optic_dr(void** p, int n, int batch, void* stream) {
  const long long total = (long long)n * batch;
  if (total > 0)
    ref_optic_dr_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>((float*)p[0], (float*)p[1],
                                                                                            (float*)p[2], n, total);
  return (int)cudaGetLastError();
}

FLYB_API int launch_optic(void** p, int n, int batch, float gr, float ga, float aad, void* stream) {
  RefOptic s{(float*)p[0], (float*)p[1], (float*)p[2], (float*)p[3], (float*)p[4], (float*)p[5], (float*)p[6], (float*)p[7]};
  const long long total = (long long)n * batch;
  if (total > 0)
    ref_optic_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(s, n, total, gr, ga, aad);
  return (int)cudaGetLastError();
}

FLYB_API int launch_csr(void** p, int rows, int cols, int batch, int half, void* stream) {
  const long long warps = (long long)rows * batch;
  const unsigned blocks = (unsigned)((warps + 7) / 8);
  if (blocks) {
    if (half)
      ref_csr_kernel<__half><<<blocks, 256, 0, (cudaStream_t)stream>>>((int*)p[0], (int*)p[1], (__half*)p[2], (float*)p[3],
                                                                       (float*)p[4], rows, cols, batch);
    else
      ref_csr_kernel<float><<<blocks, 256, 0, (cudaStream_t)stream>>>((int*)p[0], (int*)p[1], (float*)p[2], (float*)p[3],
                                                                      (float*)p[4], rows, cols, batch);
  }
  return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ the unit update of the extended substep
namespace flyb {
struct OpticUnitK {
  int m, batch, classes, mode;
  float ga, aad, norm, lo, hi;
  float scale[FLYB_SLOW_MAX_CLASSES], decay[FLYB_SLOW_MAX_CLASSES];
  float *v, *adapt, *g_slow;
  float* g_cls[FLYB_SLOW_MAX_CLASSES];
  const float* held[FLYB_SLOW_MAX_CLASSES];
  const float* rec_slow[FLYB_SLOW_MAX_CLASSES];
  const float *rec, *pr, *spk, *dr, *a;
};

// One thread per (unit, fly), the reference's operation order (optic.py:534-551).
__global__ void __launch_bounds__(256) optic_unit_kernel(OpticUnitK k) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)k.m * k.batch) return;
  const int i = (int)(t / k.batch);
  float tone = 0.0f;
  for (int c = 0; c < k.classes; ++c) {
    float target = k.held[c] ? k.held[c][t] : 0.0f;
    if (k.rec_slow[c]) target = target + k.rec_slow[c][t];
    const float ts = target * k.scale[c];
    const float gk = ts + (k.g_cls[c][t] - ts) * k.decay[c];
    k.g_cls[c][t] = gk;
    tone = tone + gk;
  }
  const float ad = k.adapt[t];
  float inp;
  if (!k.classes) {                     // the plain order (optic.py:530-532)
    inp = (k.rec[t] + k.pr[t]) - k.ga * ad;
    inp = inp + k.spk[t];
  } else if (k.mode == FLYB_SLOW_GAIN) {
    k.g_slow[t] = tone;
    const float syn = (k.rec[t] + k.pr[t]) + k.spk[t];
    float f = 1.0f + tone / k.norm;
    f = fminf(fmaxf(f, k.lo), k.hi);
    inp = syn * f - k.ga * ad;
  } else {
    k.g_slow[t] = tone;
    const float syn = (k.rec[t] + k.pr[t]) + k.spk[t];
    inp = syn - k.ga * ad;
    if (k.mode == FLYB_SLOW_ADDITIVE) inp = inp + tone;
  }
  const float v = k.v[t];
  k.v[t] = inp + (v - inp) * k.a[i];
  const float dr = k.dr[t];
  k.adapt[t] = dr + (ad - dr) * k.aad;
}
}  // namespace flyb

FLYB_API int flyb_optic_unit_step(const flyb_optic_unit_args* a, void* stream) {
  using namespace flyb;
  if (!a || a->m <= 0 || a->batch <= 0 || a->classes < 0 || a->classes > FLYB_SLOW_MAX_CLASSES || !a->v ||
      !a->adapt || !a->rec || !a->pr || !a->spk || !a->dr || !a->a)
    return FLYB_EINVAL;
  if (a->classes && (a->mode < FLYB_SLOW_ADDITIVE || a->mode > FLYB_SLOW_THRESHOLD || !a->g_slow ||
                     !(a->norm != 0.0f)))
    return FLYB_EINVAL;
  const long long total = (long long)a->m * a->batch;
  if (total >= (1ll << 31)) return FLYB_ETOOBIG;
  OpticUnitK k;
  k.m = a->m; k.batch = a->batch; k.classes = a->classes; k.mode = a->mode;
  k.ga = a->adapt_gain; k.aad = a->a_ad; k.norm = a->norm; k.lo = a->clip_lo; k.hi = a->clip_hi;
  for (int c = 0; c < FLYB_SLOW_MAX_CLASSES; ++c) {
    const bool used = c < a->classes;
    if (used && !a->g_cls[c]) return FLYB_EINVAL;
    k.scale[c] = used ? a->scale[c] : 0.0f;
    k.decay[c] = used ? a->decay[c] : 0.0f;
    k.g_cls[c] = used ? a->g_cls[c] : nullptr;
    k.held[c] = used ? a->held[c] : nullptr;
    k.rec_slow[c] = used ? a->rec_slow[c] : nullptr;
  }
  k.v = a->v; k.adapt = a->adapt; k.g_slow = a->g_slow;
  k.rec = a->rec; k.pr = a->pr; k.spk = a->spk; k.dr = a->dr; k.a = a->a;
  optic_unit_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(k);
  return (int)cudaGetLastError();
}
