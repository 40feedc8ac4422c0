// Readouts either side of the brain step: motor group means (flyverse/motor.py:232-270 through
// neural.cu:133-144) and the photoreceptor stage of the optic frame (flyverse/optic.py:496-517);
// plus the library's version / ABI / occupancy queries.
#include "common.cuh"

namespace flyb {

// Fixed-order double accumulation per (fly, group), batch-major rates (neural.cu:133-140).
__global__ void ref_means_kernel(const int* __restrict__ ptr, const int* __restrict__ idx, const float* __restrict__ rates,
                                 double* out, int n, int groups, int batch, int stride) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)groups * batch) return;
  const int b = (int)(t / groups), k = (int)(t - (long long)b * groups);
  double sum = 0.0;
  for (int j = ptr[k]; j < ptr[k + 1]; ++j) sum += (double)rates[(size_t)b * n + idx[j]];
  const int count = ptr[k + 1] - ptr[k];
  out[(size_t)b * stride + k] = count ? sum / count : 0.0;
}

// Native-layout motor readout: rates are [n][batch] (fly-minor); thread (k, b) sums group k of fly b
// in member order in double, so consecutive threads of a group read consecutive flies.
__global__ void group_means_kernel(const int* __restrict__ ptr, const int* __restrict__ idx,
                                   const float* __restrict__ rates, double* out, int groups, int batch) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)groups * batch) return;
  const int k = (int)(t / batch), b = (int)(t - (long long)k * batch);
  double sum = 0.0;
  for (int j = ptr[k]; j < ptr[k + 1]; ++j) sum += (double)rates[(size_t)idx[j] * batch + b];
  const int count = ptr[k + 1] - ptr[k];
  out[(size_t)b * groups + k] = count ? sum / count : 0.0;
}

struct PhotoK {
  int n_pr, n_col, batch;
  const float* __restrict__ rad; const int* __restrict__ pr_column; const float* __restrict__ sens;
  const int* __restrict__ avg_ptr; const int* __restrict__ avg_idx; const float* __restrict__ avg_w;
  const int* __restrict__ pr_cell; const unsigned char* __restrict__ has;
  float* I_lp; float* I_mean; float* contrast; unsigned char* fresh;
  float a_lp, c_lp, a_ad, c_ad, eps, clip_hi;
  float* a_pr;
};

// One thread per (fly, column x family cell): photoreceptor intensities of the cell's members,
// their mean, the low-pass / adaptation update and the clipped contrast (optic.py:503-513).
__global__ void photo_cell_kernel(PhotoK k) {
  const int cells = k.n_col * 5;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)cells * k.batch) return;
  const int b = (int)(t / cells), c = (int)(t - (long long)b * cells);
  const float* rb = k.rad + (size_t)b * k.n_col * 4;
  float I = 0.0f;
  for (int e = k.avg_ptr[c]; e < k.avg_ptr[c + 1]; ++e) {
    const int p = k.avg_idx[e];
    const float* r = rb + (size_t)k.pr_column[p] * 4;
    const float* s = k.sens + (size_t)p * 4;
    float ip = r[0] * s[0];
    float q = r[1] * s[1]; ip = ip + q;
    q = r[2] * s[2]; ip = ip + q;
    q = r[3] * s[3]; ip = ip + q;
    const float term = k.avg_w[e] * ip;
    I = I + term;
  }
  const size_t o = (size_t)b * cells + c;
  float lp = k.I_lp[o], mean = k.I_mean[o];
  if (k.fresh[b]) { lp = I; mean = I; }
  float x = k.a_lp * lp, y = k.c_lp * I;
  lp = x + y;
  x = k.a_ad * mean; y = k.c_ad * lp;
  mean = x + y;
  k.I_lp[o] = lp;
  k.I_mean[o] = mean;
  float num = lp - mean, den = mean + k.eps;
  float con = num / den;
  con = con < -1.0f ? -1.0f : (con > k.clip_hi ? k.clip_hi : con);
  k.contrast[o] = k.has[c] ? con : 0.0f;
}

// Gather of the contrast of each photoreceptor's cell, fly-minor; clears the fresh flags.
__global__ void photo_gather_kernel(PhotoK k) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)k.n_pr * k.batch) return;
  const int p = (int)(t / k.batch), b = (int)(t - (long long)p * k.batch);
  k.a_pr[t] = k.contrast[(size_t)b * k.n_col * 5 + k.pr_cell[p]];
  if (p == 0) k.fresh[b] = 0;
}

// One thread waits on a flag that nothing sets; the bounded wait gives up and records the error.
__global__ void selftest_wait_kernel(const int* flag, int* status, long long spins) {
  if (threadIdx.x == 0 && blockIdx.x == 0) bounded_wait_ne(flag, 0, status, spins, 2, -1);
}

// Gather-rate probe: half-warps (16 lanes x float4) read random 256-byte rows x[idx[e]][0:64] of an
// L2-resident array, 8 rows in flight per half-warp, and sum them. The access pattern of the optic
// substep at 64 flies without its arithmetic: its rate bounds that kernel from above.
__global__ void __launch_bounds__(256) gather_probe_kernel(const float4* __restrict__ x, int rows,
                                                           const int* __restrict__ idx, int n_idx, float* out) {
  constexpr int U = 8;
  const int lane = threadIdx.x & 31, sub = lane >> 4, l = lane & 15;
  const long long hw = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2 + sub;
  const long long nhw = (long long)gridDim.x * blockDim.x / 16;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (long long e0 = hw; e0 < n_idx; e0 += nhw * U) {
    int r[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const long long e = e0 + (long long)u * nhw;
      const int v = e < n_idx ? __ldg(&idx[e]) : -1;
      r[u] = (v >= 0 && v < rows) ? v : -1;
    }
    float4 v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = r[u] >= 0 ? __ldg(&x[(size_t)r[u] * 16 + l]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int u = 0; u < U; ++u) { acc.x += v[u].x; acc.y += v[u].y; acc.z += v[u].z; acc.w += v[u].w; }
  }
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = acc.x + acc.y + acc.z + acc.w;
}

int lif_blocks_per_sm(int block);
int optic_blocks_per_sm();
int adjoint_blocks_per_sm();

}  // namespace flyb

using namespace flyb;

FLYB_API int launch_means(void** p, int n, int groups, int batch, int stride, void* stream) {
  const long long total = (long long)groups * batch;
  if (total > 0)
    ref_means_kernel<<<(unsigned)((total + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        (int*)p[0], (int*)p[1], (float*)p[2], (double*)p[3], n, groups, batch, stride);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_group_means(const int* ptr, const int* idx, const float* rates, double* out, int groups, int batch,
                              void* stream) {
  if (!ptr || !rates || !out || groups < 0 || batch <= 0) return FLYB_EINVAL;
  const long long total = (long long)groups * batch;
  if (total >= (1ll << 31)) return FLYB_ETOOBIG;
  if (total)
    group_means_kernel<<<(unsigned)((total + 127) / 128), 128, 0, (cudaStream_t)stream>>>(ptr, idx, rates, out, groups,
                                                                                          batch);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_photoreceptor(const flyb_photo_args* a, void* stream) {
  if (!a || a->n_pr < 0 || a->n_col <= 0 || a->batch <= 0 || !a->rad || !a->pr_column || !a->sens || !a->avg_ptr ||
      !a->avg_idx || !a->avg_w || !a->pr_cell || !a->has || !a->I_lp || !a->I_mean || !a->contrast || !a->fresh ||
      !a->a_pr)
    return FLYB_EINVAL;
  PhotoK k{a->n_pr, a->n_col, a->batch, a->rad, a->pr_column, a->sens, a->avg_ptr, a->avg_idx, a->avg_w, a->pr_cell,
           a->has, a->I_lp, a->I_mean, a->contrast, a->fresh, a->a_lp, a->c_lp, a->a_ad, a->c_ad, a->eps, a->clip_hi,
           a->a_pr};
  cudaStream_t st = (cudaStream_t)stream;
  const long long cells = (long long)a->n_col * 5 * a->batch;
  photo_cell_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(k);
  FLYB_CHECK_LAUNCH();
  const long long prs = (long long)a->n_pr * a->batch;
  if (prs > 0) photo_gather_kernel<<<(unsigned)((prs + 255) / 256), 256, 0, st>>>(k);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_occupancy(int kind, int block, int* sm_count, int* blocks_per_sm) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (sm_count) cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev);
  int b = 0;
  if (kind == 0) b = lif_blocks_per_sm(block ? block : 256);
  else if (kind == 1) b = optic_blocks_per_sm();
  else if (kind == 2) b = adjoint_blocks_per_sm();
  else return FLYB_EINVAL;
  if (blocks_per_sm) *blocks_per_sm = b;
  return (int)cudaGetLastError();
}

FLYB_API int flyb_gather_probe(const float* x, int rows, const int* idx, int n_idx, float* out, int blocks_per_sm,
                               void* stream) {
  if (!x || !idx || !out || rows <= 0 || n_idx < 0 || blocks_per_sm < 1 || blocks_per_sm > 16) return FLYB_EINVAL;
  if (reinterpret_cast<uintptr_t>(x) & 15) return FLYB_EINVAL;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  gather_probe_kernel<<<sms * blocks_per_sm, 256, 0, (cudaStream_t)stream>>>((const float4*)x, rows, idx, n_idx, out);
  return (int)cudaGetLastError();
}

FLYB_API int flyb_selftest_wait(const int* flag, int* status, long long spins, void* stream) {
  if (!flag || !status || spins < 0) return FLYB_EINVAL;
  selftest_wait_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(flag, status, spins);
  return (int)cudaGetLastError();
}

FLYB_API const char* flyb_version(void) { return "flyb200 0.1.0 (sm_100a)"; }

FLYB_API int flyb_abi_sizes(int* sizes, int n) {
  const int s[7] = {(int)sizeof(flyb_lif_args),     (int)sizeof(flyb_optic_args), (int)sizeof(flyb_spmm_args),
                    (int)sizeof(flyb_adjoint_args), (int)sizeof(flyb_photo_args), (int)sizeof(flyb_trace_args),
                    (int)sizeof(flyb_optic_unit_args)};
  int k = 0;
  for (; k < n && k < 7; ++k) sizes[k] = s[k];
  return k;
}
