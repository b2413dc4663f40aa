// diag.cu -- device diagnostics of the reference's output routines, computed
// where the data already is (HBM); only the result crosses to the host.
//
//   pic_average_x        Average_x profiles (In-Output/Output_To_Tecplot_IJK_2D.f90:
//                        166-226): the mean of each node field over the nodes of
//                        one mesh column x = x_i, in the file's output scaling.
//   pic_energy_spectrum  Output_Energy.f90:41-71: per-species counts of the
//                        particle energy (eV) in (E_max (b-1)/N, E_max b/N] and
//                        of vx in (V_max (b-1-N/2)/N, V_max (b-N/2)/N].
//   pic_velocity_moments OUTPUT_velocity.f90:48-103: per x-column (floor(X))
//                        particle counts, drift velocity (mean) and thermal
//                        velocity (standard deviation), two passes.
//
// Counts are integers and bit-exact.  The column means sum each column in the
// reference's node order (j ascending) one thread per column, so they are
// bit-exact too.  The velocity sums are FP64 atomics (the reference sums in
// FP32, sequentially): their order, and so their last bits, vary run to run.
// Compiled with --fmad=false like the rest of the library: the absolute
// position rebuilt from a mixed-precision particle equals the one the
// download path writes.
#include <algorithm>
#include <vector>

#include "pic_ctx.h"

namespace pic {

namespace {

constexpr int kMaxProfileCols = 3 + 3 * PIC_MAX_SPECIES;

struct ProfK {
  const double *f[kMaxProfileCols];  // null: the column's x coordinate
  double scale[kMaxProfileCols];
  int ncols, nnx, nny;
  const double *xs;
  double *out;  // [ncols][nnx]
};

// Output_To_Tecplot_IJK_2D.f90:184-215: a column's nodes in node order,
// summed, divided by their count, then scaled for the file (:220-223).
__global__ void k_average_x(ProfK k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (i >= k.nnx || c >= k.ncols) return;
  double v;
  if (!k.f[c]) {
    v = k.xs[i] * k.scale[c];
  } else {
    const double *col = k.f[c] + (size_t)i * k.nny;
    double s = 0.0;
#pragma unroll 8
    for (int j = 0; j < k.nny; ++j) s = s + col[j];
    v = (s / (double)k.nny) * k.scale[c];
  }
  k.out[(size_t)c * k.nnx + i] = v;
}

// One species' particle arrays; FP32 data in the first half of the double
// storage when f32 (x, y then hold the offsets inside the element loc).
struct PartK {
  const double *x, *vx, *vy, *vz;
  const int32_t *loc;
  int64_t n;
  int f32;
  int ney;
  double xmin, hx;
};

__device__ __forceinline__ double vget(const double *a, int f32, int64_t p) {
  return f32 ? (double)reinterpret_cast<const float *>(a)[p] : a[p];
}

// absolute x of a live particle, as the download path writes it
__device__ __forceinline__ double xget(const PartK &s, int64_t p, int e) {
  if (!s.f32) return s.x[p];
  const int i = e / s.ney;
  return s.xmin + ((double)i + (double)reinterpret_cast<const float *>(s.x)[p]) * s.hx;
}

// reference bin edges, evaluated in the reference's order
__device__ __forceinline__ double e_edge(double e_max, int i, int n) { return (e_max * (double)i) / (double)n; }
__device__ __forceinline__ double v_edge(double v_max, int i, int n) {
  return (v_max * (double)((float)i - 0.5f * (float)n)) / (double)n;
}

// the bin b (0-based) of (edge[b], edge[b+1]] that holds v, or -1.  t is
// v's position in bin widths from edge[0] (a product with a reciprocal, good
// to a few ulps); the candidate and its two neighbours are checked against
// the exact edges.
__device__ __forceinline__ int find_bin(double v, double t, const double *edge, int n) {
  if (!(t > -2.0) || !(t < n + 2.0)) return -1;
  const int b0 = (int)floor(t);
  for (int b = max(b0 - 1, 0); b <= min(b0 + 1, n - 1); ++b)
    if (v <= edge[b + 1] && v > edge[b]) return b;
  return -1;
}

// add 1 to sh[bin] for every lane with bin >= 0, one shared atomic per
// distinct bin in the warp; all 32 lanes call it
__device__ __forceinline__ void warp_count(unsigned int *sh, int bin) {
  const unsigned same = __match_any_sync(0xffffffffu, bin);
  const int lane = threadIdx.x & 31;
  if (bin >= 0 && lane == __ffs(same) - 1) atomicAdd(&sh[bin], (unsigned)__popc(same));
}

struct SpecK {
  PartK s;
  int nbins;
  double mass, vref, e_max, v_max;
  double e_inv, v_inv;  // nbins / e_max, nbins / v_max
  unsigned long long *ce, *cv;
};

// Output_Energy.f90:55-71 for one species.  The grid-stride loop runs the
// same number of iterations on every lane of a warp (the base index is
// uniform), so the whole-warp match is legal.
__global__ void __launch_bounds__(256) k_spectrum(SpecK k) {
  extern __shared__ double edges[];  // [nbins+1] energy, [nbins+1] vx edges, then [2][nbins] counts
  double *ee = edges, *ve = edges + k.nbins + 1;
  unsigned int *sh = reinterpret_cast<unsigned int *>(edges + 2 * (k.nbins + 1));
  for (int b = threadIdx.x; b <= k.nbins; b += blockDim.x) {
    ee[b] = e_edge(k.e_max, b, k.nbins);
    ve[b] = v_edge(k.v_max, b, k.nbins);
  }
  for (int b = threadIdx.x; b < 2 * k.nbins; b += blockDim.x) sh[b] = 0u;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < k.s.n; base += stride) {
    const int64_t p = base + threadIdx.x;
    int be = -1, bv = -1;
    if (p < k.s.n && k.s.loc[p] >= 0) {
      const double vx = vget(k.s.vx, k.s.f32, p), vy = vget(k.s.vy, k.s.f32, p), vz = vget(k.s.vz, k.s.f32, p);
      // ParticleOne.f90:235-244 EnergyParticleOne with VFactor, then / JtoeV
      const double e = ((((0.5 * k.mass) * ((vx * vx + vy * vy) + vz * vz)) * k.vref) * k.vref) / PIC_JTOEV;
      be = find_bin(e, e * k.e_inv, ee, k.nbins);
      bv = find_bin(vx, vx * k.v_inv + 0.5 * k.nbins, ve, k.nbins);
    }
    warp_count(sh, be);
    warp_count(sh + k.nbins, bv);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < k.nbins; b += blockDim.x) {
    if (sh[b]) atomicAdd(k.ce + b, (unsigned long long)sh[b]);
    if (sh[k.nbins + b]) atomicAdd(k.cv + b, (unsigned long long)sh[k.nbins + b]);
  }
}

struct MomK {
  PartK s;
  int nbins;
  unsigned long long *count;  // [nbins]
  double *sum;                // [3][nbins] velocity sums, then variance sums
  const double *drift;        // [3][nbins] (second pass)
};

__device__ __forceinline__ int x_bin(double X, int nbins) {
  // OUTPUT_velocity.f90:57 num = MIN(MAX(1, FLOOR(X)+1), N), 0-based here
  const double f = floor(X);
  if (!(f >= 0.0)) return 0;
  if (f >= (double)(nbins - 1)) return nbins - 1;
  return (int)f;
}

// pass 1 (OUTPUT_velocity.f90:55-63): count and velocity sums per column;
// pass 2 (:80-87, kSecond): sums of (v - drift)^2
template <bool kSecond>
__global__ void __launch_bounds__(256) k_vmoments(MomK k) {
  extern __shared__ double shd[];  // [3][nbins] sums, then [3][nbins] drift (pass 2) or [nbins] counts
  double *acc = shd;
  double *dr = shd + 3 * k.nbins;
  unsigned int *cnt = reinterpret_cast<unsigned int *>(shd + 3 * k.nbins);
  for (int b = threadIdx.x; b < 3 * k.nbins; b += blockDim.x) {
    acc[b] = 0.0;
    if (kSecond) dr[b] = k.drift[b];
  }
  if (!kSecond)
    for (int b = threadIdx.x; b < k.nbins; b += blockDim.x) cnt[b] = 0u;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < k.s.n; base += stride) {
    const int64_t p = base + threadIdx.x;
    int b = -1;
    double v[3] = {0.0, 0.0, 0.0};
    if (p < k.s.n) {
      const int e = k.s.loc[p];
      if (e >= 0) {
        b = x_bin(xget(k.s, p, e), k.nbins);
        v[0] = vget(k.s.vx, k.s.f32, p);
        v[1] = vget(k.s.vy, k.s.f32, p);
        v[2] = vget(k.s.vz, k.s.f32, p);
      }
    }
    if (!kSecond) warp_count(cnt, b);
    double t[3];
    for (int c = 0; c < 3; ++c) {
      t[c] = v[c];
      if (kSecond && b >= 0) {
        const double d = v[c] - dr[c * k.nbins + b];
        t[c] = d * d;
      }
    }
    // particles sorted by cell: a warp's particles fall in one x column, or
    // in two when a column edge (one Debye length, about one cell) crosses
    // their cells.  Then the warp sums per column first and adds once per
    // column and component; otherwise every lane adds its own.  Every lane
    // takes part in each ballot and shuffle (none is skipped by
    // short-circuiting).
    const unsigned full = 0xffffffffu;
    const int b0 = __shfl_sync(full, b, 0);
    const unsigned m0 = __ballot_sync(full, b == b0);
    const int src1 = (m0 == full) ? 0 : __ffs(~m0) - 1;
    const int b1 = __shfl_sync(full, b, src1);
    const unsigned m1 = __ballot_sync(full, b == b1);
    if ((m0 | m1) == full) {
      for (int c = 0; c < 3; ++c) {
        double s0 = (b == b0) ? t[c] : 0.0, s1 = (b == b1 && b1 != b0) ? t[c] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
          s0 += __shfl_xor_sync(full, s0, o);
          s1 += __shfl_xor_sync(full, s1, o);
        }
        if ((threadIdx.x & 31) == 0) {
          if (b0 >= 0) atomicAdd(&acc[c * k.nbins + b0], s0);
          if (b1 != b0 && b1 >= 0) atomicAdd(&acc[c * k.nbins + b1], s1);
        }
      }
    } else if (b >= 0) {
      for (int c = 0; c < 3; ++c) atomicAdd(&acc[c * k.nbins + b], t[c]);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 3 * k.nbins; b += blockDim.x)
    if (acc[b] != 0.0) atomicAdd(&k.sum[b], acc[b]);
  if (!kSecond)
    for (int b = threadIdx.x; b < k.nbins; b += blockDim.x)
      if (cnt[b]) atomicAdd(&k.count[b], (unsigned long long)cnt[b]);
}

// OUTPUT_velocity.f90:64-76 (drift = sum / count, 0 for an empty column) and
// :88-103 (thermal = sqrt(variance sum / count))
__global__ void k_vmoments_div(const unsigned long long *count, const double *sum, double *out, int nbins, int root) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * nbins) return;
  const unsigned long long c = count[t % nbins];
  double v = 0.0;
  if (c != 0ull) {
    v = sum[t] / (double)c;
    if (root) v = sqrt(v);
  }
  out[t] = v;
}

PartK part_k(const Species &s) {
  PartK p;
  p.x = s.x;
  p.vx = s.vx;
  p.vy = s.vy;
  p.vz = s.vz;
  p.loc = s.loc;
  p.n = s.n_slots;
  p.f32 = s.f32 ? 1 : 0;
  p.ney = g.m.ney;
  p.xmin = g.m.xmin;
  p.hx = g.m.hx;
  return p;
}

unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(blocks_for(n, 256), 148 * 4)); }

// device scratch for the diagnostics, grown on demand and freed at finalize
struct DiagScratch {
  void *p = nullptr;
  size_t bytes = 0;
} g_diag;

int scratch(size_t bytes, void **out) {
  if (bytes > g_diag.bytes) {
    if (g_diag.p) cudaFree(g_diag.p);
    g_diag.p = nullptr;
    g_diag.bytes = 0;
    PIC_CUDA(cudaMalloc(&g_diag.p, bytes));
    g_diag.bytes = bytes;
  }
  *out = g_diag.p;
  return PIC_OK;
}

}  // namespace

void diag_free() {
  if (g_diag.p) cudaFree(g_diag.p);
  g_diag.p = nullptr;
  g_diag.bytes = 0;
}

}  // namespace pic

using namespace pic;

extern "C" {

int pic_average_x(double *out) {
  if (!g.inited) {
    set_error("pic_average_x: library not initialised (pic_init)");
    return PIC_ERR_STATE;
  }
  if (int rc = fields_fence(0x3u)) return rc;  // reads rho and phi: after a queued upload
  if (!out) {
    set_error("pic_average_x: null output");
    return PIC_ERR_ARG;
  }
  ProfK k;
  std::memset(&k, 0, sizeof k);
  // the file's columns (Output_To_Tecplot_IJK_2D.f90:219-223): x, Phi, Rho,
  // Rho_s per species, Ek_s per species, Ek_tot per species
  int c = 0;
  auto col = [&](const double *f, double scale) {
    k.f[c] = f;
    k.scale[c] = scale;
    ++c;
  };
  col(nullptr, g.L_ref);
  col(g.d_phi, g.phi_ref);
  col(g.d_rho, g.P.n_ref);
  for (int s = 0; s < g.ns; ++s) col(g.sp[s].rho_s, g.P.n_ref);
  for (int s = 0; s < g.ns; ++s) col(g.sp[s].ek_s, 1.0);
  for (int s = 0; s < g.ns; ++s) col(g.sp[s].ek_tot, 1.0);
  k.ncols = c;
  k.nnx = g.m.nnx;
  k.nny = g.m.nny;
  k.xs = g.d_xs;
  int rc;
  void *d = nullptr;
  const size_t bytes = (size_t)c * g.m.nnx * sizeof(double);
  if ((rc = scratch(bytes, &d))) return rc;
  k.out = static_cast<double *>(d);
  k_average_x<<<dim3((g.m.nnx + 127) / 128, c), 128, 0, g.st>>>(k);
  PIC_LAUNCHED();
  PIC_CUDA(cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  return PIC_OK;
}

int pic_energy_spectrum(int32_t species, int32_t nbins, double e_max_ev, double v_max, int64_t *count_e,
                        int64_t *count_vx) {
  if (!g.inited) {
    set_error("pic_energy_spectrum: library not initialised (pic_init)");
    return PIC_ERR_STATE;
  }
  if (species < 0 || species >= g.ns || nbins < 1 || nbins > 4096 || !(e_max_ev > 0) || !(v_max > 0) ||
      !count_e || !count_vx) {
    set_error("pic_energy_spectrum: bad arguments");
    return PIC_ERR_ARG;
  }
  const Species &s = g.sp[species];
  int rc;
  void *d = nullptr;
  const size_t bytes = 2 * (size_t)nbins * sizeof(unsigned long long);
  if ((rc = scratch(bytes, &d))) return rc;
  unsigned long long *cnt = static_cast<unsigned long long *>(d);
  PIC_CUDA(cudaMemsetAsync(cnt, 0, bytes, g.st));
  if (s.n_slots > 0) {
    SpecK k{part_k(s), nbins, s.mass, g.v_ref, e_max_ev, v_max, nbins / e_max_ev, nbins / v_max, cnt, cnt + nbins};
    const size_t shb = 2 * (nbins + 1) * sizeof(double) + 2 * nbins * sizeof(unsigned int);
    PIC_CUDA(cudaFuncSetAttribute(k_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shb));
    k_spectrum<<<grid_for(s.n_slots), 256, shb, g.st>>>(k);
    PIC_LAUNCHED();
  }
  std::vector<unsigned long long> h(2 * (size_t)nbins);
  PIC_CUDA(cudaMemcpyAsync(h.data(), cnt, bytes, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  for (int b = 0; b < nbins; ++b) {
    count_e[b] = (int64_t)h[b];
    count_vx[b] = (int64_t)h[nbins + b];
  }
  return PIC_OK;
}

int pic_velocity_moments(int32_t species, int32_t nbins, int64_t *count, double *drift, double *thermal) {
  if (!g.inited) {
    set_error("pic_velocity_moments: library not initialised (pic_init)");
    return PIC_ERR_STATE;
  }
  if (species < 0 || species >= g.ns || nbins < 1 || nbins > 2048 || !count || !drift || !thermal) {
    set_error("pic_velocity_moments: bad arguments");
    return PIC_ERR_ARG;
  }
  const Species &s = g.sp[species];
  const size_t nb = (size_t)nbins;
  // count [nb] u64, sums [3nb], drift [3nb], thermal [3nb]
  int rc;
  void *d = nullptr;
  if ((rc = scratch(nb * 8 * 10, &d))) return rc;
  unsigned long long *cnt = static_cast<unsigned long long *>(d);
  double *sum = reinterpret_cast<double *>(cnt + nb), *dr = sum + 3 * nb, *th = dr + 3 * nb;
  PIC_CUDA(cudaMemsetAsync(d, 0, nb * 8 * 4, g.st));
  const size_t sh1 = 3 * nb * sizeof(double) + nb * sizeof(unsigned int), sh2 = 6 * nb * sizeof(double);
  PIC_CUDA(cudaFuncSetAttribute(k_vmoments<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh1));
  PIC_CUDA(cudaFuncSetAttribute(k_vmoments<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh2));
  MomK k{part_k(s), nbins, cnt, sum, dr};
  const unsigned grid = grid_for(s.n_slots), gdiv = (unsigned)((3 * nb + 255) / 256);
  if (s.n_slots > 0) {
    k_vmoments<false><<<grid, 256, sh1, g.st>>>(k);
    PIC_LAUNCHED();
  }
  k_vmoments_div<<<gdiv, 256, 0, g.st>>>(cnt, sum, dr, nbins, 0);
  PIC_LAUNCHED();
  PIC_CUDA(cudaMemsetAsync(sum, 0, 3 * nb * sizeof(double), g.st));
  if (s.n_slots > 0) {
    k_vmoments<true><<<grid, 256, sh2, g.st>>>(k);
    PIC_LAUNCHED();
  }
  k_vmoments_div<<<gdiv, 256, 0, g.st>>>(cnt, sum, th, nbins, 1);
  PIC_LAUNCHED();
  std::vector<unsigned long long> hc(nb);
  PIC_CUDA(cudaMemcpyAsync(hc.data(), cnt, nb * 8, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaMemcpyAsync(drift, dr, 3 * nb * 8, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaMemcpyAsync(thermal, th, 3 * nb * 8, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  for (size_t b = 0; b < nb; ++b) count[b] = (int64_t)hc[b];
  return PIC_OK;
}

}  // extern "C"
