// The sensory ray tracer of the fly's eye: spheres/ellipsoids, axis-aligned boxes and planes, one
// point light with hard shadows, ambient light, procedural patterns and value-noise detail, four
// spectral channels [UV, B, G, R] (flyverse/world.py:162-300, flyverse/batch_world.py:89-147).
//
// One thread per ray. A block traces rays of one scene: the packed scene (a few KB) is staged in
// shared memory once per block and every lane reads the same primitive at the same time
// (broadcast). The shadow ray stops at the first primitive nearer than the light, which decides
// `lit` exactly as the reference's nearest-hit comparison does. With an eye (`samples` > 1) the
// block holds whole columns, and each column's weighted sample sum is formed in shared memory in
// sample order, so the per-column radiance leaves the kernel without a (B, rays, 4) round trip.
//
// Arithmetic follows the reference's tensor expressions operation by operation (the library is
// built with --fmad=false, so every product and sum is rounded on its own); the one fused form is
// the vector length, which the reference's CPU norm evaluates as a fused multiply-add chain.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "flyb200.h"

namespace {

constexpr float kInf = 1e9f;      // world.py INF
constexpr float kEps = 1e-4f;     // self-intersection margin of every primitive
constexpr float kTiny = 1e-9f;    // division guard of box slabs and planes
constexpr int kMatFloats = 16;    // refl 4, refl2 4, emit 4, pattern scale, pattern id, 2 spare
constexpr int kLightFloats = 12;  // position 3, colour 4, ambient 4, 1 spare
constexpr int kMaxObjects = 512;
#ifndef FLYB_TRACE_THREADS
#define FLYB_TRACE_THREADS 256
#endif
constexpr int kThreads = FLYB_TRACE_THREADS;  // rays per block

__host__ __device__ inline int scene_floats(int ns, int nb, int np) {
  return 6 * (ns + nb + np) + kMatFloats * (ns + nb + np + 1) + kLightFloats;
}

__device__ __forceinline__ float norm3(float x, float y, float z) {
  return sqrtf(fmaf(z, z, fmaf(y, y, x * x)));
}

// torch.remainder on floats: fmod, moved to the divisor's sign
__device__ __forceinline__ float py_mod(float a, float b) {
  float r = fmodf(a, b);
  if (r != 0.f && ((r < 0.f) != (b < 0.f))) r += b;
  return r;
}

// x mod (2^31 - 1) for 0 <= x < 2^62
__device__ __forceinline__ long long mod_mersenne31(unsigned long long x) {
  const unsigned long long m = 2147483647ull;
  x = (x & m) + (x >> 31);
  x = (x & m) + (x >> 31);
  return (long long)(x >= m ? x - m : x);
}

// second stage of the lattice hash from the first residue h in [0, 2^31 - 1)
__device__ __forceinline__ float hash_tail(long long h) {
  h = mod_mersenne31((unsigned long long)(h ^ (h >> 13)) * 1274126177ull);
  return (float)(int)(h & 65535) / 32768.0f - 1.0f;  // h >= 0
}

// lattice hash in [-1, 1] (world.py:21-25); the linear form wraps in 64 bits like torch's int64
__device__ __forceinline__ float lattice_hash(long long lin) {
  long long h = lin % 2147483647ll;
  if (h < 0) h += 2147483647ll;
  return hash_tail(h);
}

// x mod (2^31 - 1), non-negative, for |x| < 2^62: 2^31 is 1 modulo 2^31 - 1, so the high and low
// halves fold together
__device__ __forceinline__ long long residue_m31(long long x) {
  const long long m = 2147483647ll;
  x = (x >> 31) + (x & m);
  x = (x >> 31) + (x & m);
  if (x < 0) x += m;
  if (x >= m) x -= m;
  return x;
}

// int64 of an integer-valued float, through the 32-bit conversion when it fits
__device__ __forceinline__ long long to_int64(float f) {
  return fabsf(f) < 2147483648.f ? (long long)(int)f : (long long)f;
}

// trilinear value noise at period `scale` (world.py:28-43), corners in (dx, dy, dz) order
__device__ float value_noise(float px, float py, float pz, float scale) {
  const float qx = px / scale, qy = py / scale, qz = pz / scale;
  const float flx = floorf(qx), fly = floorf(qy), flz = floorf(qz);
  const long long ix = to_int64(flx), iy = to_int64(fly), iz = to_int64(flz);
  // floor() is integer valued, so converting it to int64 and back returns it unchanged
  float fx = qx - flx, fy = qy - fly, fz = qz - flz;
  fx = (fx * fx) * (3.f - 2.f * fx);
  fy = (fy * fy) * (3.f - 2.f * fy);
  fz = (fz * fz) * (3.f - 2.f * fz);
  float out = 0.f;
  if (fabsf(flx) < 1073741824.f && fabsf(fly) < 1073741824.f && fabsf(flz) < 1073741824.f) {
    // |i| < 2^30: the linear form cannot wrap, so its residue is the sum of the per-axis residues;
    // the z coefficient is the modulus itself, so z drops out and corners (x, y, 0), (x, y, 1)
    // share one hash
    const long long m = 2147483647ll;
    long long hx[2], hy[2];
    hx[0] = residue_m31(ix * 374761393ll);
    hy[0] = residue_m31(iy * 668265263ll);
    hx[1] = hx[0] + 374761393ll >= m ? hx[0] + 374761393ll - m : hx[0] + 374761393ll;
    hy[1] = hy[0] + 668265263ll >= m ? hy[0] + 668265263ll - m : hy[0] + 668265263ll;
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
      const float wx = dx ? fx : 1.f - fx;
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
        const float wy = dy ? fy : 1.f - fy;
        const long long h = hx[dx] + hy[dy];
        const float g = hash_tail(h >= m ? h - m : h);
        out = out + ((wx * wy) * (1.f - fz)) * g;
        out = out + ((wx * wy) * fz) * g;
      }
    }
    return out;
  }
  const unsigned long long A = 374761393ull, Bc = 668265263ull, C = 2147483647ull;
  const unsigned long long base = (unsigned long long)ix * A + (unsigned long long)iy * Bc + (unsigned long long)iz * C;
#pragma unroll
  for (int dx = 0; dx < 2; ++dx) {
    const float wx = dx ? fx : 1.f - fx;
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const float wy = dy ? fy : 1.f - fy;
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        const float wz = dz ? fz : 1.f - fz;
        const unsigned long long lin = base + (dx ? A : 0ull) + (dy ? Bc : 0ull) + (dz ? C : 0ull);
        out = out + ((wx * wy) * wz) * lattice_hash((long long)lin);
      }
    }
  }
  return out;
}

struct SceneSm {
  int ns, nb, np;
  const float* sph;    // [ns][6] centre, radii
  const float* box;    // [nb][6] lo, hi
  const float* pln;    // [np][6] point, unit normal
  const float* mat;    // [ns + nb + np + 1][16]
  const float* light;  // [12]
  const float* occ;    // [ns][4] per-sphere (o - c) / r and |(o - c) / r|^2 - 1 for a shared origin, or null
  const int* shadow_order;  // spheres enclosing the light first: the likeliest blockers of a shadow ray
};

struct Hit {
  float t, nx, ny, nz;
  int id;
};

__device__ __forceinline__ float sphere_t(const float* s, const float* occ, float ox, float oy, float oz, float dx,
                                          float dy, float dz) {
  float ocx, ocy, ocz, c;
  if (occ) {
    ocx = occ[0], ocy = occ[1], ocz = occ[2], c = occ[3];
  } else {
    ocx = (ox - s[0]) / s[3], ocy = (oy - s[1]) / s[4], ocz = (oz - s[2]) / s[5];
    c = ((ocx * ocx + ocy * ocy) + ocz * ocz) - 1.f;
  }
  const float ddx = dx / s[3], ddy = dy / s[4], ddz = dz / s[5];
  const float a = (ddx * ddx + ddy * ddy) + ddz * ddz;
  const float b = 2.f * ((ocx * ddx + ocy * ddy) + ocz * ddz);
  const float disc = b * b - (4.f * a) * c;
  // the reference's where(disc > 0 & t > eps, t, INF) with t = t0 > eps ? t0 : t1, evaluating
  // the square root and each quotient only where the result depends on it
  if (!(disc > 0.f)) return kInf;
  const float sq = sqrtf(disc);
  const float t0 = (-b - sq) / (2.f * a);
  if (t0 > kEps) return t0;
  const float t1 = (-b + sq) / (2.f * a);
  return t1 > kEps ? t1 : kInf;
}

__device__ __forceinline__ float box_t(const float* bx, float ox, float oy, float oz, float ix, float iy, float iz,
                                       int* axis) {
  const float lx = (bx[0] - ox) * ix, ly = (bx[1] - oy) * iy, lz = (bx[2] - oz) * iz;
  const float hx = (bx[3] - ox) * ix, hy = (bx[4] - oy) * iy, hz = (bx[5] - oz) * iz;
  float enter = fminf(lx, hx);
  int ax = 0;
  const float ny = fminf(ly, hy), nz = fminf(lz, hz);
  if (ny > enter) enter = ny, ax = 1;
  if (nz > enter) enter = nz, ax = 2;
  const float leave = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fmaxf(lz, hz));
  *axis = ax;
  return (leave > enter && enter > kEps) ? enter : kInf;
}

__device__ __forceinline__ float plane_t(const float* pl, float ox, float oy, float oz, float dx, float dy, float dz,
                                         float* denom_out) {
  const float denom = (dx * pl[3] + dy * pl[4]) + dz * pl[5];
  const float num = ((pl[0] - ox) * pl[3] + (pl[1] - oy) * pl[4]) + (pl[2] - oz) * pl[5];
  *denom_out = denom;
  // t = num / denom > eps > 0 needs |denom| > tiny and num, denom of one sign; only then divide
  if (!(fabsf(denom) > kTiny) || !((num > 0.f && denom > 0.f) || (num < 0.f && denom < 0.f))) return kInf;
  const float t = num / denom;
  return t > kEps ? t : kInf;
}

__device__ __forceinline__ float guard(float d) { return fabsf(d) < kTiny ? kTiny : d; }

// nearest hit over spheres, boxes, planes; ties keep the earliest primitive (world.py:162-211)
__device__ Hit nearest(const SceneSm& s, float ox, float oy, float oz, float dx, float dy, float dz) {
  Hit h{kInf, 0.f, 0.f, 0.f, s.ns + s.nb + s.np};
  float best = kInf;
  int k_best = -1;
  for (int k = 0; k < s.ns; ++k) {
    const float t = sphere_t(s.sph + 6 * k, s.occ ? s.occ + 4 * k : nullptr, ox, oy, oz, dx, dy, dz);
    if (t < best) best = t, k_best = k;
  }
  if (best < h.t) {
    const float* sp = s.sph + 6 * k_best;
    const float px = ox + dx * best, py = oy + dy * best, pz = oz + dz * best;
    const float nx = (px - sp[0]) / (sp[3] * sp[3]), ny = (py - sp[1]) / (sp[4] * sp[4]),
                nz = (pz - sp[2]) / (sp[5] * sp[5]);
    const float len = fmaxf(norm3(nx, ny, nz), kTiny);
    h = Hit{best, nx / len, ny / len, nz / len, k_best};
  }
  if (s.nb) {
    const float ix = 1.f / guard(dx), iy = 1.f / guard(dy), iz = 1.f / guard(dz);
    best = kInf, k_best = -1;
    int ax_best = 0;
    for (int k = 0; k < s.nb; ++k) {
      int ax;
      const float t = box_t(s.box + 6 * k, ox, oy, oz, ix, iy, iz, &ax);
      if (t < best) best = t, k_best = k, ax_best = ax;
    }
    if (best < h.t) {
      const float d = ax_best == 0 ? dx : (ax_best == 1 ? dy : dz);
      const float sign = -(d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f));
      h = Hit{best, ax_best == 0 ? sign : 0.f, ax_best == 1 ? sign : 0.f, ax_best == 2 ? sign : 0.f, s.ns + k_best};
    }
  }
  if (s.np) {
    best = kInf, k_best = -1;
    float denom_best = 0.f;
    for (int k = 0; k < s.np; ++k) {
      float denom;
      const float t = plane_t(s.pln + 6 * k, ox, oy, oz, dx, dy, dz, &denom);
      if (t < best) best = t, k_best = k, denom_best = denom;
    }
    if (best < h.t) {
      const float* pl = s.pln + 6 * k_best;
      const float flip = denom_best > 0.f ? -1.f : 1.f;
      h = Hit{best, flip * pl[3], flip * pl[4], flip * pl[5], s.ns + s.nb + k_best};
    }
  }
  return h;
}

// 1 when nothing lies nearer than `dist` along the shadow ray (world.py:276-277: ts >= dist)
__device__ float unshadowed(const SceneSm& s, float ox, float oy, float oz, float dx, float dy, float dz, float dist) {
  for (int q = 0; q < s.ns; ++q) {
    const int k = s.shadow_order[q];
    if (sphere_t(s.sph + 6 * k, nullptr, ox, oy, oz, dx, dy, dz) < dist) return 0.f;
  }
  if (s.nb) {
    const float ix = 1.f / guard(dx), iy = 1.f / guard(dy), iz = 1.f / guard(dz);
    for (int k = 0; k < s.nb; ++k) {
      int ax;
      if (box_t(s.box + 6 * k, ox, oy, oz, ix, iy, iz, &ax) < dist) return 0.f;
    }
  }
  for (int k = 0; k < s.np; ++k) {
    float denom;
    if (plane_t(s.pln + 6 * k, ox, oy, oz, dx, dy, dz, &denom) < dist) return 0.f;
  }
  // the nearest hit is INF when nothing is hit: lit only if INF >= dist as well
  return kInf >= dist ? 1.f : 0.f;
}

// shade one ray (world.py:264-300)
__device__ float4 shade(const SceneSm& s, float detail, float ox, float oy, float oz, float dx, float dy, float dz) {
  const Hit h = nearest(s, ox, oy, oz, dx, dy, dz);
  if (!(h.t < kInf)) return make_float4(0.f, 0.f, 0.f, 0.f);
  const float px = ox + dx * h.t, py = oy + dy * h.t, pz = oz + dz * h.t;
  const float* L = s.light;
  const float tx = L[0] - px, ty = L[1] - py, tz = L[2] - pz;
  const float dist = norm3(tx, ty, tz);
  const float dd = fmaxf(dist, kTiny);
  const float lx = tx / dd, ly = ty / dd, lz = tz / dd;
  const float lam = fmaxf((h.nx * lx + h.ny * ly) + h.nz * lz, 0.f);
  const float lit = unshadowed(s, px + h.nx * 1e-3f, py + h.ny * 1e-3f, pz + h.nz * 1e-3f, lx, ly, lz, dist);
  const float falloff = 4.f / (1.f + dist * dist);
  const float* m = s.mat + kMatFloats * h.id;
  // procedural pattern (world.py:281-300)
  const float sc = m[12];
  const int pat = (int)m[13];
  const float fx = floorf(px / sc), fy = floorf(py / sc);
  bool second = false;
  if (pat == 1) second = py_mod(fx + fy, 2.f) == 1.f;
  else if (pat == 2) second = py_mod(fabsf(h.nx) > 0.5f ? fy : fx, 2.f) == 1.f;
  else if (pat == 3) second = py_mod(fy, 2.f) == 1.f || py_mod(fx + 3.f * fy, 7.f) == 0.f;
  const float* r = second ? m + 4 : m;
  float mult = 1.f;
  bool detailed = detail > 0.f;
  if (detailed) {
    const float n1 = 0.5f * value_noise(px, py, pz, 0.02f);
    const float n2 = 0.3f * value_noise(px, py, pz, 0.008f);
    const float n3 = 0.2f * value_noise(px, py, pz, 0.003f);
    mult = fmaxf(1.f + detail * ((n1 + n2) + n3), 0.1f);
  }
  const float shine = (lam * lit) * falloff;
  float out[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float refl = detailed ? r[c] * mult : r[c];
    out[c] = refl * (L[7 + c] + L[3 + c] * shine) + m[8 + c];
  }
  return make_float4(out[0], out[1], out[2], out[3]);
}

struct TraceK {
  int batch, rays, samples, ns, nb, np, shared_origin, floats, outputs, per_block;
  float detail;
  const float* scene;
  const float* origins;
  const float* dirs;
  const double* eye_dirs;
  const double* pose;
  const float* weights;
  float* out;
};

__global__ void __launch_bounds__(kThreads) trace_kernel(TraceK k) {
  extern __shared__ float4 smem4[];
  float* sm = reinterpret_cast<float*>(smem4);
  const int b = blockIdx.y;
  const float* src = k.scene + (size_t)b * k.floats;
  for (int i = threadIdx.x; i < k.floats; i += blockDim.x) sm[i] = src[i];
  float* occ = sm + ((k.floats + 3) & ~3);            // [ns][4], 16-byte aligned
  float4* partial = reinterpret_cast<float4*>(occ + 4 * k.ns);
  int* order = reinterpret_cast<int*>(partial + (k.samples > 1 ? kThreads : 0));  // [ns]
  int* arrived = order + k.ns;                        // [per_block] samples finished per column
  if (k.samples > 1)
    for (int i = threadIdx.x; i < k.per_block; i += blockDim.x) arrived[i] = 0;
  SceneSm s;
  s.ns = k.ns, s.nb = k.nb, s.np = k.np;
  s.sph = sm, s.box = sm + 6 * k.ns, s.pln = sm + 6 * (k.ns + k.nb);
  s.mat = sm + 6 * (k.ns + k.nb + k.np);
  s.light = s.mat + kMatFloats * (k.ns + k.nb + k.np + 1);
  s.occ = nullptr;
  s.shadow_order = order;
  __syncthreads();
  if (threadIdx.x == 0) {
    // any order finds "some primitive nearer than the light" equally; enclosing spheres first
    const float* L = s.light;
    int q = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int i = 0; i < k.ns; ++i) {
        const float* sp = s.sph + 6 * i;
        const float ex = (L[0] - sp[0]) / sp[3], ey = (L[1] - sp[1]) / sp[4], ez = (L[2] - sp[2]) / sp[5];
        const bool encloses = (ex * ex + ey * ey) + ez * ez < 1.f;
        if (encloses == (pass == 0)) order[q++] = i;
      }
  }
  float ox = 0.f, oy = 0.f, oz = 0.f;
  if (k.shared_origin) {
    ox = k.origins[3 * b], oy = k.origins[3 * b + 1], oz = k.origins[3 * b + 2];
    for (int i = threadIdx.x; i < k.ns; i += blockDim.x) {
      const float* sp = s.sph + 6 * i;
      const float x = (ox - sp[0]) / sp[3], y = (oy - sp[1]) / sp[4], z = (oz - sp[2]) / sp[5];
      occ[4 * i] = x, occ[4 * i + 1] = y, occ[4 * i + 2] = z, occ[4 * i + 3] = ((x * x + y * y) + z * z) - 1.f;
    }
    s.occ = occ;
  }
  __syncthreads();
  const int local = threadIdx.x / k.samples, j = threadIdx.x - local * k.samples;
  const int col = blockIdx.x * k.per_block + local;
  const bool active = local < k.per_block && col < k.outputs;
  float4 rad = make_float4(0.f, 0.f, 0.f, 0.f);
  if (active) {
    const long long ray = (long long)col * k.samples + j;
    float dx, dy, dz;
    if (k.pose) {
      const double* e = k.eye_dirs + 3 * ray;
      const double* P = k.pose + 9 * b;              // forward, left, up
      dx = (float)((e[0] * P[0] + e[1] * P[3]) + e[2] * P[6]);
      dy = (float)((e[0] * P[1] + e[1] * P[4]) + e[2] * P[7]);
      dz = (float)((e[0] * P[2] + e[1] * P[5]) + e[2] * P[8]);
    } else {
      const float* d = k.dirs + 3 * ((size_t)b * k.rays + ray);
      dx = d[0], dy = d[1], dz = d[2];
    }
    if (!k.shared_origin) {
      const float* o = k.origins + 3 * ((size_t)b * k.rays + ray);
      ox = o[0], oy = o[1], oz = o[2];
    }
    rad = shade(s, k.detail, ox, oy, oz, dx, dy, dz);
  }
  float4* dst = reinterpret_cast<float4*>(k.out) + (size_t)b * k.outputs;
  if (k.samples == 1) {
    if (active) dst[col] = rad;
    return;
  }
  if (!active) return;
  // the last sample of a column to finish sums the column in sample order: no block barrier, so
  // a warp of cheap rays does not wait for the block's slowest one
  partial[threadIdx.x] = rad;
  __threadfence_block();
  if (atomicAdd(&arrived[local], 1) != k.samples - 1) return;
  __threadfence_block();
  const int first = local * k.samples;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int q = 0; q < k.samples; ++q) {
    const float w = k.weights[q];
    const float4 v = partial[first + q];
    acc.x = acc.x + v.x * w, acc.y = acc.y + v.y * w, acc.z = acc.z + v.z * w, acc.w = acc.w + v.w * w;
  }
  dst[col] = acc;
}

}  // namespace

FLYB_API int flyb_trace_scene_floats(int n_sph, int n_box, int n_pln) {
  if (n_sph < 0 || n_box < 0 || n_pln < 0 || n_sph + n_box + n_pln > kMaxObjects) return -1;
  return scene_floats(n_sph, n_box, n_pln);
}

FLYB_API int flyb_trace(const flyb_trace_args* a, void* stream) {
  if (!a || a->batch <= 0 || a->rays < 0 || a->samples < 1 || a->samples > kThreads || a->n_sph < 0 || a->n_box < 0 ||
      a->n_pln < 0)
    return FLYB_EINVAL;
  if (!a->rays) return 0;  // nothing to trace; empty outputs may have no address
  if (!a->scene || !a->out || !a->origins) return FLYB_EINVAL;
  if (a->n_sph + a->n_box + a->n_pln > kMaxObjects) return FLYB_ETOOBIG;
  if (reinterpret_cast<uintptr_t>(a->out) & 15) return FLYB_EINVAL;  // float4 stores
  if (a->rays % a->samples || (a->samples > 1 && !a->weights) || (a->pose ? !a->eye_dirs : !a->dirs) ||
      (a->pose && !a->shared_origin) || !(a->detail >= 0.f))
    return FLYB_EINVAL;
  if (a->batch > 65535 || (long long)a->batch * a->rays * 3 >= (1ll << 40)) return FLYB_ETOOBIG;
  TraceK k;
  k.batch = a->batch, k.rays = a->rays, k.samples = a->samples;
  k.ns = a->n_sph, k.nb = a->n_box, k.np = a->n_pln, k.shared_origin = a->shared_origin ? 1 : 0;
  k.floats = scene_floats(k.ns, k.nb, k.np);
  k.outputs = a->rays / a->samples;
  k.per_block = kThreads / a->samples;
  k.detail = a->detail;
  k.scene = a->scene, k.origins = a->origins, k.dirs = a->dirs, k.eye_dirs = a->eye_dirs, k.pose = a->pose;
  k.weights = a->weights, k.out = a->out;
  // scene (rounded up to 16 bytes), per-sphere origin terms, per-thread radiance for the sample sums
  const size_t bytes = (size_t)(((k.floats + 3) & ~3) + 4 * k.ns) * sizeof(float) +
                       (a->samples > 1 ? kThreads * sizeof(float4) : 0) + (size_t)(k.ns + k.per_block) * sizeof(int);
  if (bytes > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(trace_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
  }
  const dim3 grid((unsigned)((k.outputs + k.per_block - 1) / k.per_block), (unsigned)k.batch);
  trace_kernel<<<grid, kThreads, bytes, (cudaStream_t)stream>>>(k);
  return (int)cudaGetLastError();
}
