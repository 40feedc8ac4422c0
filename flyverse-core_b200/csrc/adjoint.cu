// Hand-written adjoint of the optic-lobe rate dynamics (forward: flyverse/optic.py:525-551), for
// gradients with respect to per-type-pair gains and per-type time constants. The reference has
// no adjoint; its gradients come from torch autograd through optic.py:606-676.
//
// Forward substep t (per unit i, fly b; W = W_rr with gains folded in):
//   dr_t = clip(v_t + b, 0, 1) - b
//   inp_t = gr * (W dr_t) + pr - ga * adapt_t + spk
//   v_{t+1} = inp_t + (v_t - inp_t) * a          adapt_{t+1} = dr_t + (adapt_t - dr_t) * aad
// Reverse step, with lam_v = dL/dv_{t+1}, lam_a = dL/dadapt_{t+1}, m_t = 1[0 <= v_t + b <= 1]
// (the derivative torch assigns to clamp):
//   mu_t      = (1 - a) * lam_v
//   dL/dv_t   = a * lam_v + m_t * (gr * (W^T mu_t) + (1 - aad) * lam_a)
//   dL/dad_t  = aad * lam_a - ga * mu_t
//   g_edge[e] += mu_t[i] * dr_t[j]        for e = (i <- j): dL/dW_ij = gr * g_edge[e]
//   g_a[i]    += lam_v[i] * (v_t[i] - inp_t[i])   (dL/da_i)
// W^T is walked as the CSR of the transpose: warp w owns transposed rows j (presynaptic units),
// so the per-edge accumulator g_edge, g_a[j] and the in-place lam updates of row j have a single
// writer. mu is double-buffered, so one grid barrier per reverse step suffices.
#include "common.cuh"

namespace flyb {

struct AdjK {
  int m, batch, nsteps;
  const int* __restrict__ t_ptr; const int* __restrict__ t_col; const float* __restrict__ t_w;
  const int* __restrict__ t_perm;
  const float* __restrict__ v_hist; const float* __restrict__ inp_hist;
  const float* __restrict__ a; const float* __restrict__ b;
  float gr, ga, aad;
  float* lam_v; float* lam_a;
  float* mu0; float* mu1;
  float* g_edge; float* g_a;
  int* status; int* sync;
};

// Phase 1 for the rows of this warp: mu_t = (1 - a) lam_v and the g_a accumulation.
template <int F, int FPL>
__device__ __forceinline__ void adj_phase1(const AdjK& k, int t, float* mu, long long warp0, long long nwarps) {
  const int lane = threadIdx.x & 31;
  const size_t sz = (size_t)k.m * k.batch;
  for (long long j = warp0; j < k.m; j += nwarps) {
    float part = 0.0f;
    if (lane < F) {
      const float aj = k.a[j];
      const float oma = 1.0f - aj;
#pragma unroll
      for (int q = 0; q < FPL; ++q) {
        const int bb = lane * FPL + q;
        if (bb < k.batch) {
          const size_t e = (size_t)j * k.batch + bb;
          const float lv = k.lam_v[e];
          mu[e] = oma * lv;
          const float d = k.v_hist[(size_t)t * sz + e] - k.inp_hist[(size_t)t * sz + e];
          part = part + lv * d;
        }
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) part = part + __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) k.g_a[j] = k.g_a[j] + part;
  }
}

// Phase 2: z = W^T mu over transposed row j, the lam updates and the per-edge accumulation.
template <int F, int FPL>
__device__ __forceinline__ void adj_phase2(const AdjK& k, int t, const float* __restrict__ mu, long long warp0,
                                           long long nwarps) {
  constexpr int G = 32 / F;
  const int lane = threadIdx.x & 31, g = lane / F, f = lane % F, fb = f * FPL;
  const size_t sz = (size_t)k.m * k.batch;
  for (long long j = warp0; j < k.m; j += nwarps) {
    const float bj = k.b[j];
    float dr[FPL];
#pragma unroll
    for (int q = 0; q < FPL; ++q) {
      const int bb = fb + q;
      dr[q] = bb < k.batch ? clip01(k.v_hist[(size_t)t * sz + (size_t)j * k.batch + bb] + bj) - bj : 0.0f;
    }
    float acc[FPL];
#pragma unroll
    for (int q = 0; q < FPL; ++q) acc[q] = 0.0f;
    constexpr int U = FPL <= 2 ? 8 : (FPL == 4 ? 4 : 2);
    const int e0 = k.t_ptr[j], e1 = k.t_ptr[j + 1];
    // lane group g takes entries e0 + g + G*k; U gathers of mu in flight per lane
    for (int base = e0 + g; base - g < e1; base += G * U) {
      int ii[U];
      float ww[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = base + u * G;
        const bool ok = e < e1;
        ii[u] = ok ? __ldg(&k.t_col[e]) : -1;
        ww[u] = ok ? __ldg(&k.t_w[e]) : 0.0f;
      }
      float mv[U][FPL];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < FPL; ++q)
          mv[u][q] = (ii[u] >= 0 && fb + q < k.batch) ? mu[(size_t)ii[u] * k.batch + fb + q] : 0.0f;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        float ge = 0.0f;
#pragma unroll
        for (int q = 0; q < FPL; ++q) {
          const float p = ww[u] * mv[u][q];
          acc[q] = acc[q] + p;
          const float pg = mv[u][q] * dr[q];
          ge = ge + pg;
        }
        // sum the per-edge term over the F lanes of this group (every lane takes part)
#pragma unroll
        for (int o = 1; o < F; o <<= 1) ge = ge + __shfl_xor_sync(0xffffffffu, ge, o);
        if (ii[u] >= 0 && f == 0) {
          const int ee = base + u * G;
          const int pe = k.t_perm ? k.t_perm[ee] : ee;
          k.g_edge[pe] = k.g_edge[pe] + ge;
        }
      }
    }
#pragma unroll
    for (int o = F; o < 32; o <<= 1)
#pragma unroll
      for (int q = 0; q < FPL; ++q) acc[q] = acc[q] + __shfl_xor_sync(0xffffffffu, acc[q], o);
    if (lane < F) {
      const float aj = k.a[j];
      const float omaad = 1.0f - k.aad;
#pragma unroll
      for (int q = 0; q < FPL; ++q) {
        const int bb = lane * FPL + q;
        if (bb < k.batch) {
          const size_t e = (size_t)j * k.batch + bb;
          const float x = k.v_hist[(size_t)t * sz + e] + bj;
          const float mask = (x >= 0.0f && x <= 1.0f) ? 1.0f : 0.0f;
          const float lv = k.lam_v[e], la = k.lam_a[e];
          float inner = k.gr * acc[q];
          inner = inner + omaad * la;
          float nl = aj * lv;
          nl = nl + mask * inner;
          k.lam_v[e] = nl;
          float na = k.aad * la;
          na = na - k.ga * mu[e];
          k.lam_a[e] = na;
        }
      }
    }
  }
}

template <int F, int FPL>
__global__ void __launch_bounds__(256) adj_phase1_kernel(AdjK k, int t) {
  float* mu = (t & 1) ? k.mu1 : k.mu0;
  adj_phase1<F, FPL>(k, t, mu, ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                     ((long long)gridDim.x * blockDim.x) >> 5);
}

template <int F, int FPL>
__global__ void __launch_bounds__(256) adj_phase2_kernel(AdjK k, int t) {
  const float* mu = (t & 1) ? k.mu1 : k.mu0;
  adj_phase2<F, FPL>(k, t, mu, ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                     ((long long)gridDim.x * blockDim.x) >> 5);
}

template <int F, int FPL>
__global__ void __launch_bounds__(256) adj_persistent_kernel(AdjK k) {
  int generation = 0;
  const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (int t = k.nsteps - 1; t >= 0; --t) {
    float* mu = (t & 1) ? k.mu1 : k.mu0;
    adj_phase1<F, FPL>(k, t, mu, w0, nw);
    if (!grid_barrier(k.sync, k.status, generation, t)) return;
    adj_phase2<F, FPL>(k, t, mu, w0, nw);
  }
}

template <int F, int FPL>
static int run_adjoint(const AdjK& k, int launch, int grid_cap, cudaStream_t st) {
  const unsigned blocks = (unsigned)((k.m + 7) / 8);
  if (launch == FLYB_LAUNCH_STEP) {
    for (int t = k.nsteps - 1; t >= 0; --t) {
      adj_phase1_kernel<F, FPL><<<blocks, 256, 0, st>>>(k, t);
      FLYB_CHECK_LAUNCH();
      adj_phase2_kernel<F, FPL><<<blocks, 256, 0, st>>>(k, t);
      FLYB_CHECK_LAUNCH();
    }
    return 0;
  }
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adj_persistent_kernel<F, FPL>, 256, 0);
  long long grid = (long long)sms * per_sm;
  if (grid > blocks) grid = blocks;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  if (grid < 1) return FLYB_ECOOP;
  cudaError_t e = cudaMemsetAsync(k.sync, 0, 2 * sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  AdjK kk = k;
  void* args[] = {&kk};
  e = cudaLaunchCooperativeKernel((void*)adj_persistent_kernel<F, FPL>, dim3((unsigned)grid), dim3(256), args, 0, st);
  return (int)e;
}

#define FLYB_ADJ_DISPATCH(B, CALL)                                     \
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

int adjoint_blocks_per_sm() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, adj_persistent_kernel<1, 1>, 256, 0);
  return b;
}

// Segmented gather-sum for the gradient reductions: out[s] = alpha * sum over positions e of
// segment s (seg_ptr[s] <= e < seg_ptr[s + 1]) of x[idx[e]] * (w ? w[idx[e]] : 1). One warp per
// segment: lane l sums positions l, l + 32, ... in order, then a fixed butterfly; the result is
// deterministic and FP32 throughout. The pair gains' gradient is the per-edge accumulator summed
// over the edges of each pair (idx: edges grouped by pair) times gr * W0; the time constants'
// is g_a * a summed over the units of each type.
__global__ void __launch_bounds__(256) segment_sum_kernel(const int* __restrict__ seg_ptr, const int* __restrict__ idx,
                                                           const float* __restrict__ x, const float* __restrict__ w,
                                                           float alpha, float* __restrict__ out, int segments) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long s = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < segments; s += warps) {
    const int e0 = __ldg(&seg_ptr[s]), e1 = __ldg(&seg_ptr[s + 1]);
    float sum = 0.0f;
    for (int e = e0 + lane; e < e1; e += 32) {
      const int i = __ldg(&idx[e]);
      const float term = w ? __ldg(&x[i]) * __ldg(&w[i]) : __ldg(&x[i]);
      sum = sum + term;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) sum = sum + __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) out[s] = alpha * sum;
  }
}

}  // namespace flyb

using namespace flyb;

FLYB_API int flyb_segment_sum(const int* seg_ptr, const int* idx, const float* x, const float* w, float alpha,
                              float* out, int segments, void* stream) {
  if (!seg_ptr || !idx || !x || !out || segments < 0) return FLYB_EINVAL;
  if (segments == 0) return 0;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = ((long long)segments + 7) / 8;
  if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
  segment_sum_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(seg_ptr, idx, x, w, alpha, out, segments);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_optic_adjoint(const flyb_adjoint_args* a, void* stream) {
  if (!a || a->m <= 0 || a->batch <= 0 || a->nsteps < 0 || !a->t_ptr || !a->t_col || !a->t_w || !a->v_hist ||
      !a->inp_hist || !a->a || !a->b || !a->lam_v || !a->lam_a || !a->lam_tmp || !a->mu || !a->g_edge || !a->g_a)
    return FLYB_EINVAL;
  if ((long long)a->m * a->batch >= (1ll << 31)) return FLYB_ETOOBIG;
  if (a->launch == FLYB_LAUNCH_PERSISTENT && (!a->sync || !a->status)) return FLYB_EINVAL;
  if (a->nsteps == 0) return 0;
  AdjK k{a->m, a->batch, a->nsteps, a->t_ptr, a->t_col, a->t_w, a->t_perm, a->v_hist, a->inp_hist, a->a, a->b,
         a->gr, a->ga, a->aad, a->lam_v, a->lam_a, a->mu, a->lam_tmp, a->g_edge, a->g_a, a->status, a->sync};
  cudaStream_t st = (cudaStream_t)stream;
  FLYB_ADJ_DISPATCH(a->batch, (run_adjoint<F, FPL>(k, a->launch, a->grid, st)));
}
