// unet_ops.cu -- the learned preconditioner's network kernels other than the
// tensor-core convolutions: input features, pooling, upsample + concat, ReLU
// backward, the 1x1 head, loss, output scaling, the weight gradient of the
// 3x3 convolutions, and Adam.  NHWC BF16 activations are moved 8 channels
// (16 bytes) per thread; parameters and gradients are FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/picunet.h"

namespace {

using bf16 = __nv_bfloat16;

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }
inline unsigned capped(int64_t n, int t, unsigned cap) {
  unsigned b = nblk(n, t);
  return b < cap ? (b ? b : 1u) : cap;
}

int launched() { return cudaPeekAtLastError() == cudaSuccess ? UNET_OK : UNET_ERR_CUDA; }

// 8 BF16 channels as one 16-byte word
struct V8 {
  uint4 u;
};

__device__ __forceinline__ void v8_to_f(const V8 &v, float f[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v.u);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float2 t = __bfloat1622float2(h[q]);
    f[2 * q] = t.x;
    f[2 * q + 1] = t.y;
  }
}

__device__ __forceinline__ V8 f_to_v8(const float f[8]) {
  V8 v;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v.u);
#pragma unroll
  for (int q = 0; q < 4; ++q) h[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
  return v;
}

__device__ __forceinline__ V8 ld8(const bf16 *p) { V8 v; v.u = *reinterpret_cast<const uint4 *>(p); return v; }
__device__ __forceinline__ void st8(bf16 *p, const V8 &v) { *reinterpret_cast<uint4 *>(p) = v.u; }

// ---- residual scale -------------------------------------------------------
// s = sqrt(sum over unknown nodes of r^2 / count): per-block partials in a
// fixed order; the last block to finish sums them in block order
// (deterministic), writes scale[0] = s, scale[1] = 1/s (0 when r = 0) and
// re-arms the ticket.
constexpr int RMS_THREADS = 256;

__global__ void __launch_bounds__(RMS_THREADS) k_rms(int64_t npix, const double *__restrict__ r,
                                                     const int32_t *__restrict__ mask, double *__restrict__ part,
                                                     unsigned int *ticket, double *__restrict__ scale) {
  __shared__ double ss[RMS_THREADS];
  __shared__ double sc[RMS_THREADS];
  __shared__ bool last;
  double s = 0.0, c = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * RMS_THREADS + threadIdx.x; p < npix; p += (int64_t)gridDim.x * RMS_THREADS)
    if (mask[p] > 0) {
      s += r[p] * r[p];
      c += 1.0;
    }
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  for (int o = RMS_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      sc[threadIdx.x] += sc[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ss[0];
    part[2 * blockIdx.x + 1] = sc[0];
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double ts = 0.0, tc = 0.0;
  for (unsigned b = 0; b < gridDim.x; ++b) {
    ts += *(volatile double *)&part[2 * b];
    tc += *(volatile double *)&part[2 * b + 1];
  }
  const double v = (tc > 0.0) ? sqrt(ts / tc) : 0.0;
  scale[0] = v;
  scale[1] = (v > 0.0) ? 1.0 / v : 0.0;
  *ticket = 0u;
}

__global__ void k_features(int64_t npix, const double *__restrict__ r, const double *__restrict__ scale,
                           const float *__restrict__ fs, bf16 *__restrict__ x) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  const float f[8] = {(float)(r[p] * scale[1]), fs[3 * p], fs[3 * p + 1], fs[3 * p + 2], 0.f, 0.f, 0.f, 0.f};
  st8(x + 8 * p, f_to_v8(f));
}

// ---- pooling / upsampling (g = channel group of 8) --------------------------
__global__ void k_pool(int n, int h, int w, int c, const bf16 *__restrict__ x, bf16 *__restrict__ y) {
  const int h2 = (h + 1) / 2, w2 = (w + 1) / 2, G = c / 8;
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * h2 * w2 * G) return;
  const int g = (int)(idx % G);
  const int64_t q = idx / G;
  const int j2 = (int)(q % w2), i2 = (int)((q / w2) % h2), b = (int)(q / ((int64_t)w2 * h2));
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int cnt = 0;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj) {
      const int i = 2 * i2 + di, j = 2 * j2 + dj;
      if (i < h && j < w) {
        float f[8];
        v8_to_f(ld8(x + (((int64_t)b * h + i) * w + j) * c + 8 * g), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] += f[e];
        ++cnt;
      }
    }
  const float inv = 1.0f / (float)cnt;
#pragma unroll
  for (int e = 0; e < 8; ++e) s[e] *= inv;
  st8(y + idx * 8, f_to_v8(s));
}

__global__ void k_pool_bwd(int n, int h, int w, int c, const bf16 *__restrict__ dy, bf16 *__restrict__ dx,
                           int acc) {
  const int h2 = (h + 1) / 2, w2 = (w + 1) / 2, G = c / 8;
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * h * w * G) return;
  const int g = (int)(idx % G);
  const int64_t q = idx / G;
  const int j = (int)(q % w), i = (int)((q / w) % h), b = (int)(q / ((int64_t)w * h));
  const int i2 = i / 2, j2 = j / 2;
  const float inv = 1.0f / (float)((min(2 * i2 + 2, h) - 2 * i2) * (min(2 * j2 + 2, w) - 2 * j2));
  float f[8];
  v8_to_f(ld8(dy + (((int64_t)b * h2 + i2) * w2 + j2) * c + 8 * g), f);
#pragma unroll
  for (int e = 0; e < 8; ++e) f[e] *= inv;
  if (acc) {
    float a[8];
    v8_to_f(ld8(dx + idx * 8), a);
#pragma unroll
    for (int e = 0; e < 8; ++e) f[e] += a[e];
  }
  st8(dx + idx * 8, f_to_v8(f));
}

__global__ void k_upcat(int n, int h, int w, int c1, int c2, const bf16 *__restrict__ lo,
                        const bf16 *__restrict__ skip, bf16 *__restrict__ y) {
  const int h2 = (h + 1) / 2, w2 = (w + 1) / 2, G1 = c1 / 8, G = (c1 + c2) / 8;
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * h * w * G) return;
  const int g = (int)(idx % G);
  const int64_t q = idx / G;
  const int j = (int)(q % w), i = (int)((q / w) % h), b = (int)(q / ((int64_t)w * h));
  const bf16 *src = (g < G1) ? lo + (((int64_t)b * h2 + i / 2) * w2 + j / 2) * c1 + 8 * g
                             : skip + q * c2 + 8 * (g - G1);
  st8(y + idx * 8, ld8(src));
}

__global__ void k_upcat_bwd_lo(int n, int h, int w, int c1, int c2, const bf16 *__restrict__ dy,
                               bf16 *__restrict__ dlo) {
  const int h2 = (h + 1) / 2, w2 = (w + 1) / 2, G1 = c1 / 8, ct = c1 + c2;
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * h2 * w2 * G1) return;
  const int g = (int)(idx % G1);
  const int64_t q = idx / G1;
  const int j2 = (int)(q % w2), i2 = (int)((q / w2) % h2), b = (int)(q / ((int64_t)w2 * h2));
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj) {
      const int i = 2 * i2 + di, j = 2 * j2 + dj;
      if (i < h && j < w) {
        float f[8];
        v8_to_f(ld8(dy + (((int64_t)b * h + i) * w + j) * ct + 8 * g), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] += f[e];
      }
    }
  st8(dlo + idx * 8, f_to_v8(s));
}

__global__ void k_upcat_bwd_skip(int64_t npix, int c1, int c2, const bf16 *__restrict__ dy,
                                 bf16 *__restrict__ dskip, int acc) {
  const int G2 = c2 / 8, ct = c1 + c2;
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npix * G2) return;
  const int g = (int)(idx % G2);
  const int64_t p = idx / G2;
  V8 v = ld8(dy + p * ct + c1 + 8 * g);
  if (acc) {
    float f[8], a[8];
    v8_to_f(v, f);
    v8_to_f(ld8(dskip + idx * 8), a);
#pragma unroll
    for (int e = 0; e < 8; ++e) f[e] += a[e];
    v = f_to_v8(f);
  }
  st8(dskip + idx * 8, v);
}

// ---- ReLU backward + bias gradient ------------------------------------------
// Block of G * floor(256/G) threads (G = c/8 channel groups): each thread keeps
// one channel group for the whole grid-stride loop and sums its 8 bias
// gradients in registers.
__global__ void k_relu_bwd(int64_t npix, int c, const bf16 *__restrict__ y, bf16 *__restrict__ dy,
                           float *__restrict__ db) {
  extern __shared__ float sdb[];
  const int G = c / 8;
  for (int k = threadIdx.x; k < c; k += blockDim.x) sdb[k] = 0.0f;
  __syncthreads();
  const int g = threadIdx.x % G;
  float a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t tot = npix * G;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
       idx += (int64_t)gridDim.x * blockDim.x) {
    float fy[8], fd[8];
    v8_to_f(ld8(y + idx * 8), fy);
    v8_to_f(ld8(dy + idx * 8), fd);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      fd[e] = (fy[e] > 0.0f) ? fd[e] : 0.0f;
      a[e] += fd[e];
    }
    st8(dy + idx * 8, f_to_v8(fd));
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) atomicAdd(&sdb[8 * g + e], a[e]);
  __syncthreads();
  for (int k = threadIdx.x; k < c; k += blockDim.x) atomicAdd(db + k, sdb[k]);
}

// ---- 1x1 head (c = 32) --------------------------------------------------------
__global__ void k_head(int64_t npix, const bf16 *__restrict__ y, const float *__restrict__ w,
                       const float *__restrict__ b, float *__restrict__ z) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  float s = b[0];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    float f[8];
    v8_to_f(ld8(y + p * 32 + 8 * g), f);
#pragma unroll
    for (int e = 0; e < 8; ++e) s = fmaf(w[8 * g + e], f[e], s);
  }
  z[p] = s;
}

__global__ void k_head_bwd(int64_t npix, const bf16 *__restrict__ y, const float *__restrict__ w,
                           const float *__restrict__ gz, bf16 *__restrict__ dy, float *__restrict__ dw,
                           float *__restrict__ db) {
  __shared__ float s[33];
  if (threadIdx.x < 33) s[threadIdx.x] = 0.0f;
  __syncthreads();
  float a[32], ab = 0.0f;
#pragma unroll
  for (int k = 0; k < 32; ++k) a[k] = 0.0f;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
    const float gp = gz[p];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      float f[8], o[8];
      v8_to_f(ld8(y + p * 32 + 8 * g), f);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        o[e] = gp * w[8 * g + e];
        a[8 * g + e] = fmaf(gp, f[e], a[8 * g + e]);
      }
      st8(dy + p * 32 + 8 * g, f_to_v8(o));
    }
    ab += gp;
  }
#pragma unroll
  for (int k = 0; k < 32; ++k) atomicAdd(&s[k], a[k]);
  atomicAdd(&s[32], ab);
  __syncthreads();
  if (threadIdx.x < 32) atomicAdd(dw + threadIdx.x, s[threadIdx.x]);
  if (threadIdx.x == 32) atomicAdd(db, s[32]);
}

__global__ void k_loss(int64_t npix, const float *__restrict__ z, const double *__restrict__ t,
                       const double *__restrict__ scale, const int32_t *__restrict__ mask, float *__restrict__ gz,
                       double *__restrict__ acc) {
  __shared__ double sd[2];
  if (threadIdx.x < 2) sd[threadIdx.x] = 0.0;
  __syncthreads();
  const double inv_scale = scale[1];
  double a0 = 0.0, a1 = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
    if (mask[p] > 0) {
      const double tt = t[p] * inv_scale;
      const double d = (double)z[p] - tt;
      gz[p] = (float)(2.0 * d);
      a0 += d * d;
      a1 += tt * tt;
    } else {
      gz[p] = 0.0f;
    }
  }
  atomicAdd(&sd[0], a0);
  atomicAdd(&sd[1], a1);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(acc, sd[0]);
    atomicAdd(acc + 1, sd[1]);
  }
}

__global__ void k_output(int64_t npix, const float *__restrict__ z, const double *__restrict__ scale,
                         const int32_t *__restrict__ mask, double *__restrict__ out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  out[p] = (mask[p] > 0) ? scale[0] * (double)z[p] : 0.0;
}

__global__ void k_adam(int64_t n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, bf16 *__restrict__ pb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (pb) pb[i] = __float2bfloat16(pi);
}

// Weight gradient of a 3x3 'same' convolution on the CUDA cores.  CTA =
// (32 output channels x 32 input channels) x a strided set of 32-pixel tiles;
// each thread accumulates 9 taps x 4 input channels of one output channel in
// registers, from tiles of dy and of the 9 shifted x staged in shared memory.
__global__ void __launch_bounds__(256) k_wgrad(int n, int h, int w, int c, int k, const bf16 *__restrict__ x,
                                               const bf16 *__restrict__ dy, float *__restrict__ dw) {
  __shared__ float sdy[32][33];
  __shared__ float sx[9][32][33];
  const int ncb = (c + 31) / 32;
  const int kb = blockIdx.x / ncb, cb = blockIdx.x % ncb;
  const int t = threadIdx.x;
  const int kk = t >> 3, cq = (t & 7) * 4;
  const int64_t np = (int64_t)n * h * w;
  float acc[9][4];
#pragma unroll
  for (int a = 0; a < 9; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = 0.0f;
  for (int64_t p0 = (int64_t)blockIdx.y * 32; p0 < np; p0 += (int64_t)gridDim.y * 32) {
    for (int e = t; e < 32 * 32; e += 256) {
      const int pp = e >> 5, kc = e & 31;
      const int64_t p = p0 + pp;
      const int kx = kb * 32 + kc;
      sdy[pp][kc] = (p < np && kx < k) ? __bfloat162float(dy[p * k + kx]) : 0.0f;
    }
    for (int e = t; e < 9 * 32 * 32; e += 256) {
      const int tap = e >> 10, pp = (e >> 5) & 31, cc = e & 31;
      const int64_t p = p0 + pp;
      const int cx = cb * 32 + cc;
      float v = 0.0f;
      if (p < np && cx < c) {
        const int j = (int)(p % w), i = (int)((p / w) % h);
        const int64_t b = p / ((int64_t)w * h);
        const int ii = i + tap / 3 - 1, jj = j + tap % 3 - 1;
        if (ii >= 0 && ii < h && jj >= 0 && jj < w) v = __bfloat162float(x[((b * h + ii) * w + jj) * c + cx]);
      }
      sx[tap][pp][cc] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int pp = 0; pp < 32; ++pp) {
      const float d = sdy[pp][kk];
#pragma unroll
      for (int tap = 0; tap < 9; ++tap)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[tap][q] = fmaf(d, sx[tap][pp][cq + q], acc[tap][q]);
    }
    __syncthreads();
  }
  const int kx = kb * 32 + kk;
  if (kx >= k) return;
#pragma unroll
  for (int tap = 0; tap < 9; ++tap)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int cx = cb * 32 + cq + q;
      if (cx < c && acc[tap][q] != 0.0f) atomicAdd(dw + ((int64_t)kx * 9 + tap) * c + cx, acc[tap][q]);
    }
}

__global__ void k_fill(int64_t n, float *p, float v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_tobf16(int64_t n, const float *s, bf16 *d) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = __float2bfloat16(s[i]);
}

}  // namespace

extern "C" {

int unet_rms(int64_t npix, const double *r, const int32_t *mask, double *scratch, double *scale, void *stream) {
  if (npix <= 0 || !r || !mask || !scratch || !scale) return UNET_ERR_SHAPE;
  const unsigned g = capped(npix, RMS_THREADS, UNET_RMS_BLOCKS);
  unsigned int *ticket = (unsigned int *)(scratch + 2 * UNET_RMS_BLOCKS);
  k_rms<<<g, RMS_THREADS, 0, (cudaStream_t)stream>>>(npix, r, mask, scratch, ticket, scale);
  return launched();
}

int unet_features(int32_t h, int32_t w, const double *r, const double *scale, const float *feat_static,
                  void *x_out, void *stream) {
  const int64_t np = (int64_t)h * w;
  if (np <= 0) return UNET_ERR_SHAPE;
  k_features<<<nblk(np, 256), 256, 0, (cudaStream_t)stream>>>(np, r, scale, feat_static, (bf16 *)x_out);
  return launched();
}

int unet_pool(int32_t n, int32_t h, int32_t w, int32_t c, const void *x, void *y, void *stream) {
  if (n < 1 || h < 1 || w < 1 || c < 8 || c % 8) return UNET_ERR_SHAPE;
  const int64_t tot = (int64_t)n * ((h + 1) / 2) * ((w + 1) / 2) * (c / 8);
  k_pool<<<nblk(tot, 256), 256, 0, (cudaStream_t)stream>>>(n, h, w, c, (const bf16 *)x, (bf16 *)y);
  return launched();
}

int unet_pool_bwd(int32_t n, int32_t h, int32_t w, int32_t c, const void *dy, void *dx, int32_t accumulate,
                  void *stream) {
  if (n < 1 || h < 1 || w < 1 || c < 8 || c % 8) return UNET_ERR_SHAPE;
  const int64_t tot = (int64_t)n * h * w * (c / 8);
  k_pool_bwd<<<nblk(tot, 256), 256, 0, (cudaStream_t)stream>>>(n, h, w, c, (const bf16 *)dy, (bf16 *)dx,
                                                                accumulate);
  return launched();
}

int unet_upcat(int32_t n, int32_t h, int32_t w, int32_t c1, int32_t c2, const void *lo, const void *skip,
               void *y, void *stream) {
  if (n < 1 || h < 1 || w < 1 || c1 < 8 || c2 < 8 || c1 % 8 || c2 % 8) return UNET_ERR_SHAPE;
  const int64_t tot = (int64_t)n * h * w * ((c1 + c2) / 8);
  k_upcat<<<nblk(tot, 256), 256, 0, (cudaStream_t)stream>>>(n, h, w, c1, c2, (const bf16 *)lo,
                                                             (const bf16 *)skip, (bf16 *)y);
  return launched();
}

int unet_upcat_bwd(int32_t n, int32_t h, int32_t w, int32_t c1, int32_t c2, const void *dy, void *dlo,
                   void *dskip, int32_t accumulate_skip, void *stream) {
  if (n < 1 || h < 1 || w < 1 || c1 < 8 || c2 < 8 || c1 % 8 || c2 % 8) return UNET_ERR_SHAPE;
  const int64_t tlo = (int64_t)n * ((h + 1) / 2) * ((w + 1) / 2) * (c1 / 8);
  k_upcat_bwd_lo<<<nblk(tlo, 256), 256, 0, (cudaStream_t)stream>>>(n, h, w, c1, c2, (const bf16 *)dy,
                                                                    (bf16 *)dlo);
  const int64_t npix = (int64_t)n * h * w;
  k_upcat_bwd_skip<<<nblk(npix * (c2 / 8), 256), 256, 0, (cudaStream_t)stream>>>(
      npix, c1, c2, (const bf16 *)dy, (bf16 *)dskip, accumulate_skip);
  return launched();
}

int unet_relu_bwd(int64_t npix, int32_t c, const void *y, void *dy, float *db, void *stream) {
  if (npix < 1 || c < 8 || c % 8 || c > 1024) return UNET_ERR_SHAPE;
  const int G = c / 8;
  const int threads = G * (256 / G > 0 ? 256 / G : 1);
  const unsigned g = capped(npix * G, threads, 148u * 4u);
  k_relu_bwd<<<g, threads, c * sizeof(float), (cudaStream_t)stream>>>(npix, c, (const bf16 *)y, (bf16 *)dy, db);
  return launched();
}

int unet_head(int64_t npix, int32_t c, const void *y, const float *w, const float *b, float *z, void *stream) {
  if (npix < 1 || c != 32) return UNET_ERR_SHAPE;
  k_head<<<nblk(npix, 256), 256, 0, (cudaStream_t)stream>>>(npix, (const bf16 *)y, w, b, z);
  return launched();
}

int unet_head_bwd(int64_t npix, int32_t c, const void *y, const float *w, const float *gz, void *dy, float *dw,
                  float *db, void *stream) {
  if (npix < 1 || c != 32) return UNET_ERR_SHAPE;
  k_head_bwd<<<capped(npix, 256, 148u * 4u), 256, 0, (cudaStream_t)stream>>>(npix, (const bf16 *)y, w, gz,
                                                                              (bf16 *)dy, dw, db);
  return launched();
}

int unet_loss(int64_t npix, const float *z, const double *target, const double *scale, const int32_t *mask,
              float *gz, double *loss2, void *stream) {
  if (npix < 1) return UNET_ERR_SHAPE;
  k_loss<<<capped(npix, 256, 148u * 8u), 256, 0, (cudaStream_t)stream>>>(npix, z, target, scale, mask, gz, loss2);
  return launched();
}

int unet_output(int64_t npix, const float *z, const double *scale, const int32_t *mask, double *out,
                void *stream) {
  if (npix < 1) return UNET_ERR_SHAPE;
  k_output<<<nblk(npix, 256), 256, 0, (cudaStream_t)stream>>>(npix, z, scale, mask, out);
  return launched();
}

int unet_adam(int64_t n, float *p, const float *g, float *m, float *v, void *p_bf16, float lr, float beta1,
              float beta2, float eps, int32_t t, void *stream) {
  if (n < 1 || t < 1) return UNET_ERR_SHAPE;
  const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  k_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, (bf16 *)p_bf16, lr, beta1, beta2, eps,
                                                          c1, c2);
  return launched();
}

int unet_wgrad(int32_t n, int32_t h, int32_t w, int32_t c, int32_t k, const void *x, const void *dy, float *dw,
               void *stream) {
  if (n < 1 || h < 1 || w < 1 || c < 1 || k < 1) return UNET_ERR_SHAPE;
  const int64_t np = (int64_t)n * h * w;
  const unsigned gx = (unsigned)(((k + 31) / 32) * ((c + 31) / 32));
  unsigned gy = (unsigned)((np + 31) / 32);
  const unsigned cap = (148u * 8u + gx - 1) / gx;
  if (gy > cap) gy = cap;
  k_wgrad<<<dim3(gx, gy), 256, 0, (cudaStream_t)stream>>>(n, h, w, c, k, (const bf16 *)x, (const bf16 *)dy, dw);
  return launched();
}

int unet_fill_f32(int64_t n, float *p, float v, void *stream) {
  if (n < 1) return UNET_ERR_SHAPE;
  k_fill<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, p, v);
  return launched();
}

int unet_f32_to_bf16(int64_t n, const float *src, void *dst, void *stream) {
  if (n < 1) return UNET_ERR_SHAPE;
  k_tobf16<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(n, src, (bf16 *)dst);
  return launched();
}

}  // extern "C"
