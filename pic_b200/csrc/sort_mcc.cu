// sort_mcc.cu -- counting sort of the particle SoA and MCC_jw null collisions.
//
// Counting sort: particles are ordered by element, ties by particle id, so the
// permutation is a pure function of (element, id) and the oracle reproduces it
// exactly.  Absorbed slots (loc = -1) are dropped, which replaces the
// reference's swap-with-last deletion (ParticleBundle.f90:120-127).
//
// MCC: the reference picks N = INT(NPar*P_null) (+1 with probability equal to
// the residue) distinct particles by a partial Fisher-Yates shuffle
// (mc/MCCPublic.F90:113-171).  Here every live particle gets a 32-bit key,
// a keyed hash of its id with round keys drawn from Philox per (seed, step,
// species); the N particles with the smallest (key, id) are selected.  That
// is the same law -- a uniform random N-subset -- computed with a histogram
// instead of a serial shuffle.  The collision itself
// restates mc/TypeMCC.f90:58-198, mc/MCCChi.f90, mc/MCCElectron.F90:13-148 and
// mc/MCCIon.F90:6-75 with Philox draws instead of RANDOM_NUMBER.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pic_ctx.h"
#include "pic_mcc_kin.h"

namespace pic {

// ---------------------------------------------------------------------------
// counting sort
// ---------------------------------------------------------------------------

// Runs of equal keys in a warp (particles are nearly cell-sorted): the head
// lane of each run, the run's length and each lane's rank in its run.  Equal
// keys that are not adjacent form separate runs.  Every lane takes part.
__device__ __forceinline__ void warp_runs(int key, int lane, int *head, int *len, int *rank) {
  const int prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool is_head = lane == 0 || key != prev;
  const unsigned heads = __ballot_sync(0xffffffffu, is_head);
  const unsigned upto = heads & (0xffffffffu >> (31 - lane));  // heads at lanes <= lane
  *head = 31 - __clz(upto);
  const unsigned above = lane == 31 ? 0u : heads & (0xfffffffeu << lane);  // heads after lane
  const int end = above ? __ffs(above) - 1 : 32;
  *len = end - *head;
  *rank = lane - *head;
}

// Both passes give each warp 128 consecutive slots, 32 per round: the four
// rounds' loads are issued together (a single 4-byte load per thread left
// the passes waiting on memory latency), then each round aggregates its runs.
constexpr int kSortRounds = 4;

__global__ void k_sort_count(const int32_t *__restrict__ loc, int64_t n, int32_t *__restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t wbase = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kSortRounds;
  int key[kSortRounds];
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u) {
    const int64_t p = wbase + 32 * u + lane;
    key[u] = p < n ? loc[p] : -1;
  }
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u) {
    int head, len, rank;
    warp_runs(key[u], lane, &head, &len, &rank);
    if (key[u] >= 0 && rank == 0) atomicAdd(count + key[u], len);
  }
}

// exclusive scan, 3 passes of 4096 items per block
__global__ void __launch_bounds__(1024) k_scan_block(const int32_t *in, int32_t *out, int64_t n,
                                                     int32_t *blk) {
  __shared__ int32_t s[1024];
  int64_t base = (int64_t)blockIdx.x * 4096 + threadIdx.x * 4;
  int32_t v[4], sum = 0;
  for (int k = 0; k < 4; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    sum += v[k];
  }
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int32_t t = (threadIdx.x >= off) ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  int32_t run = s[threadIdx.x] - sum;
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 1023) blk[blockIdx.x] = s[1023];
}

__global__ void k_scan_add(int32_t *out, int64_t n, const int32_t *blk_scanned) {
  int64_t i = (int64_t)blockIdx.x * 4096 + threadIdx.x;
  int32_t add = blk_scanned[blockIdx.x];
  for (int k = 0; k < 4; ++k) {
    int64_t q = i + k * 1024;
    if (q < n) out[q] += add;
  }
}

static int scan_exclusive(int32_t *in, int32_t *out, int64_t n) {
  int nb = (int)((n + 4095) / 4096);
  if (nb > 4096) {
    set_error("scan: more than 16.7M cells");
    return PIC_ERR_ARG;
  }
  k_scan_block<<<nb, 1024, 0, g.st>>>(in, out, n, g.d_scan_blk);
  PIC_LAUNCHED();
  if (nb > 1) {
    // scan the block totals in place (<= 4096 of them: one block)
    k_scan_block<<<1, 1024, 0, g.st>>>(g.d_scan_blk, g.d_scan_blk, nb, g.d_scan_blk + 4096);
    PIC_LAUNCHED();
    k_scan_add<<<nb, 1024, 0, g.st>>>(out, n, g.d_scan_blk);
    PIC_LAUNCHED();
  }
  return PIC_OK;
}

// the four rounds' cursor reservations are also in flight together
__global__ void k_sort_scatter(const int32_t *__restrict__ loc, const uint32_t *__restrict__ id, int64_t n,
                               int32_t *__restrict__ cursor, int32_t *__restrict__ perm,
                               uint32_t *__restrict__ sid) {
  const int lane = threadIdx.x & 31;
  const int64_t wbase = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kSortRounds;
  int key[kSortRounds], head[kSortRounds], len[kSortRounds], rank[kSortRounds], base[kSortRounds];
  uint32_t pid[kSortRounds];
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u) {
    const int64_t p = wbase + 32 * u + lane;
    key[u] = p < n ? loc[p] : -1;
    pid[u] = p < n ? id[p] : 0u;
  }
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u) warp_runs(key[u], lane, &head[u], &len[u], &rank[u]);
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u)
    base[u] = (key[u] >= 0 && rank[u] == 0) ? atomicAdd(cursor + key[u], len[u]) : 0;
#pragma unroll
  for (int u = 0; u < kSortRounds; ++u) {
    const int b = __shfl_sync(0xffffffffu, base[u], head[u]);
    if (key[u] >= 0) {
      const int dst = b + rank[u];
      perm[dst] = (int32_t)(wbase + 32 * u + lane);
      sid[dst] = pid[u];
    }
  }
}

// One warp per element: order its segment by id (ids are unique), writing the
// source slots to perm2.  Segments of up to 128 are ranked from shared
// memory, four ids per read (padded with the largest id, which ranks after
// every real one).
__global__ void k_sort_cells(const int32_t *__restrict__ start, int64_t ne, const int32_t *__restrict__ perm,
                             const uint32_t *__restrict__ sid, int32_t *__restrict__ perm2) {
  __shared__ __align__(16) uint32_t sh[8][128];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t c = (int64_t)blockIdx.x * 8 + warp;
  if (c >= ne) return;
  int s0 = start[c], s1 = start[c + 1], m = s1 - s0;
  if (m <= 0) return;
  if (m == 1) {
    if (lane == 0) perm2[s0] = perm[s0];
    return;
  }
  if (m <= 128) {
    const int m4 = (m + 3) & ~3;
    for (int k = lane; k < m4; k += 32) sh[warp][k] = k < m ? sid[s0 + k] : 0xffffffffu;
    __syncwarp();
    const uint4 *v = reinterpret_cast<const uint4 *>(sh[warp]);
    for (int k = lane; k < m; k += 32) {
      const uint32_t me = sh[warp][k];
      int rank = 0;
      for (int q = 0; q < m4 / 4; ++q) {
        const uint4 w = v[q];
        rank += (w.x < me) + (w.y < me) + (w.z < me) + (w.w < me);
      }
      perm2[s0 + rank] = perm[s0 + k];
    }
    return;
  }
  for (int k = lane; k < m; k += 32) {
    const uint32_t me = sid[s0 + k];
    int rank = 0;
    for (int q = 0; q < m; ++q) rank += (sid[s0 + q] < me);
    perm2[s0 + rank] = perm[s0 + k];
  }
}

template <class T>
__global__ void k_gather(const T *__restrict__ src, T *__restrict__ dst, const int32_t *__restrict__ perm,
                         int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}

// T = double (FP64 particles) or float (mixed precision: offsets in the
// element and velocities, in the first half of the same storage)
template <class T>
struct Gather7 {
  const T *x, *y, *vx, *vy, *vz;
  const int32_t *loc;
  const uint32_t *id;
  T *ox, *oy, *ovx, *ovy, *ovz;
  int32_t *oloc;
  uint32_t *oid;
};

// four particles per thread, their slot indices then all their loads issued
// together (memory-level parallelism for the scattered reads)
constexpr int kGatherItems = 4;
template <class T>
__global__ void k_gather_all(Gather7<T> g7, const int32_t *__restrict__ perm, int64_t n) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x * kGatherItems + threadIdx.x;
  int32_t p[kGatherItems];
#pragma unroll
  for (int u = 0; u < kGatherItems; ++u) {
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    p[u] = i < n ? perm[i] : -1;
  }
  T x[kGatherItems], y[kGatherItems], vx[kGatherItems], vy[kGatherItems], vz[kGatherItems];
  int32_t lc[kGatherItems];
  uint32_t id[kGatherItems];
#pragma unroll
  for (int u = 0; u < kGatherItems; ++u) {
    if (p[u] < 0) continue;
    x[u] = g7.x[p[u]];
    y[u] = g7.y[p[u]];
    vx[u] = g7.vx[p[u]];
    vy[u] = g7.vy[p[u]];
    vz[u] = g7.vz[p[u]];
    lc[u] = g7.loc[p[u]];
    id[u] = g7.id[p[u]];
  }
#pragma unroll
  for (int u = 0; u < kGatherItems; ++u) {
    if (p[u] < 0) continue;
    const int64_t i = i0 + (int64_t)u * blockDim.x;
    g7.ox[i] = x[u];
    g7.oy[i] = y[u];
    g7.ovx[i] = vx[u];
    g7.ovy[i] = vy[u];
    g7.ovz[i] = vz[u];
    g7.oloc[i] = lc[u];
    g7.oid[i] = id[u];
  }
}

int sort_species(int sidx) {
  Species &s = g.sp[sidx];
  const int64_t ne = g.ne;
  if (s.n_slots == 0) return PIC_OK;
  if (int rc_ = zero_async(g.d_cell_count, (ne + 1) * sizeof(int32_t), g.st)) return rc_;
  k_sort_count<<<blocks_for(s.n_slots, 256 * kSortRounds), 256, 0, g.st>>>(s.loc, s.n_slots, g.d_cell_count);
  PIC_LAUNCHED();
  int rc = scan_exclusive(g.d_cell_count, g.d_cell_start, ne + 1);
  if (rc) return rc;
  PIC_CUDA(cudaMemcpyAsync(g.d_cell_fill, g.d_cell_start, (ne + 1) * sizeof(int32_t),
                           cudaMemcpyDeviceToDevice, g.st));
  int32_t total = 0;
  PIC_CUDA(cudaMemcpyAsync(&total, g.d_cell_start + ne, sizeof total, cudaMemcpyDeviceToHost, g.st));
  k_sort_scatter<<<blocks_for(s.n_slots, 256 * kSortRounds), 256, 0, g.st>>>(s.loc, s.id, s.n_slots,
                                                                             g.d_cell_fill, g.d_perm, g.d_sort_id);
  PIC_LAUNCHED();
  k_sort_cells<<<blocks_for(ne, 8), 256, 0, g.st>>>(g.d_cell_start, ne, g.d_perm, g.d_sort_id, g.d_perm2);
  PIC_LAUNCHED();
  PIC_CUDA(cudaStreamSynchronize(g.st));
  if (total > 0) {
    if (s.f32) {
      auto F = [](double *v) { return reinterpret_cast<float *>(v); };
      Gather7<float> g7{F(s.x), F(s.y), F(s.vx), F(s.vy), F(s.vz), s.loc, s.id,
                        F(s.x2), F(s.y2), F(s.vx2), F(s.vy2), F(s.vz2), s.loc2, s.id2};
      k_gather_all<float><<<blocks_for(total, 256 * kGatherItems), 256, 0, g.st>>>(g7, g.d_perm2, total);
    } else {
      Gather7<double> g7{s.x, s.y, s.vx, s.vy, s.vz, s.loc, s.id, s.x2, s.y2, s.vx2, s.vy2, s.vz2, s.loc2, s.id2};
      k_gather_all<double><<<blocks_for(total, 256 * kGatherItems), 256, 0, g.st>>>(g7, g.d_perm2, total);
    }
    PIC_LAUNCHED();
  }
  std::swap(s.x, s.x2);
  std::swap(s.y, s.y2);
  std::swap(s.vx, s.vx2);
  std::swap(s.vy, s.vy2);
  std::swap(s.vz, s.vz2);
  std::swap(s.loc, s.loc2);
  std::swap(s.id, s.id2);
  s.n_slots = total;
  s.n_live = total;
  return PIC_OK;
}

// ---------------------------------------------------------------------------
// MCC
// ---------------------------------------------------------------------------

// per-species device blocks: kMccSel status words of the bounded selection
// ([0] list entries, [1] keys below the bound, [2] b*, [3] count below b*,
// [4] 1 when the selection holds) and kMccMisc counters ([0] selected below
// b*, [1] ties, [2..2+NR) reaction counts, [12] ionisations)
constexpr int kMccSel = 8;
constexpr int kMccMisc = 16;

struct MccK {
  double *x, *y, *vx, *vy, *vz;  // FP32 data in the same storage when f32
  const int32_t *loc;
  const uint32_t *id;
  int64_t n;
  uint32_t seed0, seed1, step_lo, step_hi, species;
  int f32;
  McSelect sel;  // round keys of the selection keys of this species and step
};

__device__ __forceinline__ double mcc_get(const double *a, int f32, int64_t p) {
  return f32 ? (double)reinterpret_cast<const float *>(a)[p] : a[p];
}

__device__ __forceinline__ void mcc_put(double *a, int f32, int64_t p, double v) {
  if (f32) reinterpret_cast<float *>(a)[p] = (float)v;
  else a[p] = v;
}

// Selection keys of the live particles: histogram of their top 16 bits, and
// the key itself for k_mcc_pick.
__global__ void k_mcc_hist(MccK k, uint32_t *__restrict__ hist, uint32_t *__restrict__ keys) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= k.n || k.loc[p] < 0) return;
  uint32_t key = mcc_select_key(k.id[p], k.sel);
  keys[p] = key;
  atomicAdd(hist + (key >> 16), 1u);
}

// particles below the threshold bin are selected; the threshold bin's
// particles become candidates ordered later by (key, id)
__global__ void k_mcc_pick(MccK k, const uint32_t *__restrict__ keys, uint32_t bstar, int32_t *__restrict__ sel,
                           int64_t *__restrict__ misc, uint64_t *__restrict__ cand, int32_t *__restrict__ cand_slot,
                           int64_t cand_cap) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= k.n || k.loc[p] < 0) return;
  const uint32_t key = keys[p];
  uint32_t bin = key >> 16;
  if (bin < bstar) {
    long long i = atomicAdd((unsigned long long *)&misc[0], 1ull);
    sel[i] = (int32_t)p;
  } else if (bin == bstar) {
    long long i = atomicAdd((unsigned long long *)&misc[1], 1ull);
    if (i < cand_cap) {
      cand[i] = ((uint64_t)key << 32) | (uint64_t)k.id[p];
      cand_slot[i] = (int32_t)p;
    }
  }
}

// ---- selection under a key bound: only the live particles whose key lies
// below `bound` (chosen so that about 2 ncoll + 64 of them are expected
// there) enter a 65536-bin histogram of [0, bound) and a compact list of
// (key << 32 | id, slot); the threshold bin, the particles below it and the
// order of the ties are then found on the device.  The selected set is the
// one the full histogram gives: the ncoll smallest (key, id).  When fewer
// than ncoll keys lie below the bound, or the list overflows, the host
// reruns the selection with the full histogram.

// Four consecutive slots per thread: their elements and ids come in one
// 16-byte load each, issued together and unconditionally, so every thread
// keeps 32 bytes in flight (one 4-byte load that a second one waits on left
// the pass latency-bound at a quarter of the memory bandwidth).
__global__ void k_mcc_scan(MccK k, MccSink sink) {
  const int64_t p0 = 4 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  const int lane = threadIdx.x & 31;
  int loc[4];
  uint32_t id[4];
  if (p0 + 3 < k.n) {
    const int4 l = __ldcs(reinterpret_cast<const int4 *>(k.loc + p0));
    const uint4 d = __ldcs(reinterpret_cast<const uint4 *>(k.id + p0));
    loc[0] = l.x; loc[1] = l.y; loc[2] = l.z; loc[3] = l.w;
    id[0] = d.x; id[1] = d.y; id[2] = d.z; id[3] = d.w;
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      loc[u] = p0 + u < k.n ? k.loc[p0 + u] : -1;
      id[u] = p0 + u < k.n ? k.id[p0 + u] : 0u;
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const uint32_t key = mcc_select_key(id[u], sink.rk);
    mcc_sink_put(sink, lane, loc[u] >= 0 && (uint64_t)key < sink.bound, key, id[u], p0 + u);
  }
}

// one block of 1024 threads: the bin b* where the running count of the
// histogram reaches ncoll, and the count below it.  ms[1] = keys below the
// bound, ms[2] = b* (-1 when fewer than ncoll keys lie below the bound),
// ms[3] = particles in bins below b*.  Each thread sums its 64 bins from
// sixteen 16-byte loads (eight in flight at a time); after the block scan
// warp 0 finds b* inside the one thread's 64 bins that reaches ncoll, two
// bins a lane.
__global__ void __launch_bounds__(1024) k_mcc_bstar(const uint32_t *__restrict__ hist, int64_t ncoll,
                                                    int64_t *__restrict__ ms) {
  __shared__ unsigned long long part[1024];
  __shared__ int owner;
  __shared__ unsigned long long owner_excl;
  const int t = threadIdx.x;
  if (t == 0) {
    ms[2] = -1;
    owner = -1;
  }
  const uint4 *h4 = reinterpret_cast<const uint4 *>(hist) + 16 * t;
  unsigned long long s = 0;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    uint4 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = h4[8 * half + u];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      s += (unsigned long long)v[u].x + (unsigned long long)v[u].y + (unsigned long long)v[u].z +
           (unsigned long long)v[u].w;
  }
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan
    const unsigned long long v = t >= off ? part[t - off] : 0ull;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  const unsigned long long incl = part[t], excl = t ? part[t - 1] : 0ull, nc = (unsigned long long)ncoll;
  if (t == 1023) ms[1] = (int64_t)incl;
  if (excl < nc && incl >= nc) {  // exactly one thread
    owner = t;
    owner_excl = excl;
  }
  __syncthreads();
  const int o = owner;
  if (o < 0 || t >= 32) return;
  // lane t holds bins b0 and b0 + 1 of the owner's range
  const int b0 = o * 64 + 2 * t;
  const unsigned long long h0 = hist[b0], h1 = hist[b0 + 1];
  unsigned long long x = h0 + h1;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {  // inclusive warp scan of the pairs
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, off);
    if (t >= off) x += y;
  }
  const unsigned long long before = owner_excl + x - (h0 + h1);  // keys in bins below b0
  // reached within this pair (true from the first such lane on: the last
  // lane's pair ends at the owner's inclusive count, which reaches ncoll)
  const unsigned hit = __ballot_sync(0xffffffffu, before + h0 + h1 >= nc);
  if (t == __ffs(hit) - 1) {
    if (before + h0 >= nc) {
      ms[2] = b0;
      ms[3] = (int64_t)before;
    } else {
      ms[2] = b0 + 1;
      ms[3] = (int64_t)(before + h0);
    }
  }
}

// list entries below b* are selected; those in b* are the ties
__global__ void k_mcc_pick_list(const uint64_t *__restrict__ lkey, const int32_t *__restrict__ lslot,
                                const unsigned long long *__restrict__ cnt, int64_t cap, uint64_t bound,
                                const int64_t *__restrict__ ms, int32_t *__restrict__ sel,
                                uint64_t *__restrict__ tkey, int32_t *__restrict__ tslot, int64_t tcap,
                                int64_t *__restrict__ misc) {
  const int64_t m = min((int64_t)*cnt, cap), bstar = ms[2];
  if (bstar < 0) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t kv = lkey[i];
    const int64_t bin = mcc_bin((uint32_t)(kv >> 32), bound);
    if (bin < bstar) {
      const long long j = atomicAdd((unsigned long long *)&misc[0], 1ull);
      sel[j] = lslot[i];
    } else if (bin == bstar) {
      const long long j = atomicAdd((unsigned long long *)&misc[1], 1ull);
      if (j < tcap) {
        tkey[j] = kv;
        tslot[j] = lslot[i];
      }
    }
  }
}

// one block: each tie's rank among the ties by (key, id); the first
// ncoll - below of them complete the selection.  Quadratic in the tie count,
// so it leaves more than kMaxTies ties to the full selection (a bin holds
// about 2 ncoll / 65536 keys: a few hundred at most in practice).
// Thread 0 also records in ms[4] whether the selection holds: the list did
// not overflow, b* exists, every entry below b* was picked, the ties fill
// the selection and fit their buffer and this kernel's quadratic rank.
constexpr int64_t kMaxTies = 8192;
__global__ void __launch_bounds__(1024) k_mcc_ties(const uint64_t *__restrict__ tkey,
                                                   const int32_t *__restrict__ tslot, int64_t tcap, int64_t lcap,
                                                   int64_t *__restrict__ ms, const int64_t *__restrict__ misc,
                                                   int64_t ncoll, int32_t *__restrict__ sel) {
  if (threadIdx.x == 0)
    ms[4] = (ms[0] <= lcap && ms[2] >= 0 && misc[0] == ms[3] && misc[1] >= ncoll - ms[3] && misc[1] <= tcap &&
             misc[1] <= kMaxTies)
                ? 1
                : 0;
  if (ms[2] < 0 || misc[1] > kMaxTies) return;
  const int64_t c = min(misc[1], tcap), below = ms[3], need = ncoll - below;
  for (int64_t i = threadIdx.x; i < c; i += blockDim.x) {
    const uint64_t ki = tkey[i];
    int64_t rank = 0;
    for (int64_t j = 0; j < c; ++j) rank += tkey[j] < ki ? 1 : 0;
    if (rank < need) sel[below + rank] = tslot[i];
  }
}

struct CollK {
  MccK k;
  const int32_t *sel;
  int64_t n_sel;
  const int64_t *ok;  // nullptr, or a flag that must be 1 (the bounded selection held)
  const double *prob;
  McTable tab;
  McGas gas;
  double mass, vref;
  int64_t *misc;        // [2..2+NR) reaction counts, [12] ionisations
  int64_t *ion_parent;  // (id << 32) | slot
  double *ion_data;     // 6 doubles per ionisation
  int64_t ion_cap;
};

__global__ void k_mcc_collide(CollK c) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.n_sel || (c.ok && *c.ok != 1)) return;
  int32_t p = c.sel[t];
  McParticle P;
  P.vx = mcc_get(c.k.vx, c.k.f32, p) * c.vref;
  P.vy = mcc_get(c.k.vy, c.k.f32, p) * c.vref;
  P.vz = mcc_get(c.k.vz, c.k.f32, p) * c.vref;
  McOut out;
  McRng rng;
  mc_rng_init(&rng, c.k.id[p], c.k.step_lo, c.k.step_hi, c.k.species, c.k.seed0, c.k.seed1);
  mc_collide(&P, &c.tab, c.prob, &c.gas, c.mass, &rng, &out);
  mcc_put(c.k.vx, c.k.f32, p, P.vx / c.vref);
  mcc_put(c.k.vy, c.k.f32, p, P.vy / c.vref);
  mcc_put(c.k.vz, c.k.f32, p, P.vz / c.vref);
  if (out.reaction > 0) atomicAdd((unsigned long long *)&c.misc[2 + out.reaction - 1], 1ull);
  if (out.ionised) {
    long long i = atomicAdd((unsigned long long *)&c.misc[12], 1ull);
    if (i < c.ion_cap) {
      c.ion_parent[i] = ((int64_t)c.k.id[p] << 32) | (int64_t)p;
      double *d = c.ion_data + 6 * i;
      d[0] = out.e_new[0] / c.vref;
      d[1] = out.e_new[1] / c.vref;
      d[2] = out.e_new[2] / c.vref;
      d[3] = out.ion_new[0];  // SI, converted with the ion species' factor on append
      d[4] = out.ion_new[1];
      d[5] = out.ion_new[2];
    }
  }
}

struct AppendK {
  const double *px, *py;
  const int32_t *ploc;
  double *x, *y, *vx, *vy, *vz;
  int32_t *loc;
  uint32_t *id;
  int64_t base;
  uint32_t id_base;
  const int32_t *parent_slot;  // in rank order
  const double *vel;           // 3 per created particle, normalised
  int64_t n;
  int f32;                     // both species mixed precision: FP32 offsets/velocities
};

__global__ void k_mcc_append(AppendK a) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.n) return;
  int32_t ps = a.parent_slot[r];
  int64_t d = a.base + r;
  if (a.f32) {  // the parent's element and offsets are the new particle's position
    reinterpret_cast<float *>(a.x)[d] = reinterpret_cast<const float *>(a.px)[ps];
    reinterpret_cast<float *>(a.y)[d] = reinterpret_cast<const float *>(a.py)[ps];
  } else {
    a.x[d] = a.px[ps];
    a.y[d] = a.py[ps];
  }
  mcc_put(a.vx, a.f32, d, a.vel[3 * r + 0]);
  mcc_put(a.vy, a.f32, d, a.vel[3 * r + 1]);
  mcc_put(a.vz, a.f32, d, a.vel[3 * r + 2]);
  a.loc[d] = a.ploc[ps];
  a.id[d] = a.id_base + (uint32_t)r;
}

// Rank of each ionisation of a species among the others by its parent key
// (id << 32 | slot: ids are unique, so keys are), from shared-memory tiles of
// all the keys: the created particles are appended in parent-id order, the
// order the oracle appends them in, whatever order the collisions recorded
// them in.  n^2 compares: a few thousand to some ten thousand a step.
__global__ void __launch_bounds__(128) k_ion_rank(const int64_t *__restrict__ parent, int64_t n,
                                                 int32_t *__restrict__ order) {
  __shared__ int64_t tile[2048];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t me = i < n ? parent[i] : 0;
  int64_t rank = 0;
  for (int64_t t0 = 0; t0 < n; t0 += 2048) {
    const int m = n - t0 < 2048 ? (int)(n - t0) : 2048;
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += blockDim.x) tile[k] = parent[t0 + k];
    __syncthreads();
    if (i < n)
      for (int k = 0; k < m; ++k) rank += tile[k] < me ? 1 : 0;
  }
  if (i < n) order[rank] = (int32_t)i;
}

// The appended particles' parent slots and velocities in rank order: the
// created electron's (normalised in k_mcc_collide), the ion's (SI, divided
// by v_ref here, as MCCAddNewParticle normalises it)
__global__ void k_ion_build(const int64_t *__restrict__ parent, const double *__restrict__ data,
                            const int32_t *__restrict__ order, int64_t n, double vref, int32_t *__restrict__ pslot,
                            double *__restrict__ vel_e, double *__restrict__ vel_i) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t src = order[r];
  pslot[r] = (int32_t)(parent[src] & 0xffffffff);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    vel_e[3 * r + q] = data[6 * src + q];
    vel_i[3 * r + q] = data[6 * src + 3 + q] / vref;
  }
}

// selected slots and the ionisation outputs (one region of mcc_cap entries
// per species); grown only before anything of the step is queued
static int mcc_alloc(int64_t need) {
  if (need <= g.mcc_cap) return PIC_OK;
  int64_t cap = std::max<int64_t>(need, 1 << 16);
  cudaFree(g.d_sel);
  cudaFree(g.d_ion_parent);
  cudaFree(g.d_ion_data);
  g.d_sel = nullptr;
  g.d_ion_parent = nullptr;
  g.d_ion_data = nullptr;
  g.mcc_cap = 0;
  PIC_CUDA(cudaMalloc(&g.d_sel, cap * sizeof(int32_t)));
  PIC_CUDA(cudaMalloc(&g.d_ion_parent, PIC_MAX_SPECIES * cap * sizeof(int64_t)));
  PIC_CUDA(cudaMalloc(&g.d_ion_data, PIC_MAX_SPECIES * 6 * cap * sizeof(double)));
  g.mcc_cap = cap;
  return PIC_OK;
}

// candidates of the threshold bin (key << 32 | id) and their slots; the
// caller has no queued kernel using them when they grow
static int mcc_cand_alloc(int64_t need) {
  if (need <= g.cand_cap) return PIC_OK;
  const int64_t cap = std::max<int64_t>(need, 1 << 16);
  cudaFree(g.d_cand);
  cudaFree(g.d_cand_slot);
  g.d_cand = nullptr;
  g.d_cand_slot = nullptr;
  g.cand_cap = 0;
  PIC_CUDA(cudaMalloc(&g.d_cand, cap * sizeof(uint64_t)));
  PIC_CUDA(cudaMalloc(&g.d_cand_slot, cap * sizeof(int32_t)));
  g.cand_cap = cap;
  return PIC_OK;
}

// compact list of the bounded selection and its counters (kept across steps)
static int mcc_list_alloc(int64_t need) {
  if (!g.d_msel) PIC_CUDA(cudaMalloc(&g.d_msel, PIC_MAX_SPECIES * kMccSel * sizeof(int64_t)));
  if (need <= g.mlist_cap) return PIC_OK;
  const int64_t cap = std::max<int64_t>(need + need / 2, 1 << 16);
  cudaFree(g.d_mlist_key);
  cudaFree(g.d_mlist_slot);
  g.d_mlist_key = nullptr;
  g.d_mlist_slot = nullptr;
  g.mlist_cap = 0;
  PIC_CUDA(cudaMalloc(&g.d_mlist_key, PIC_MAX_SPECIES * cap * sizeof(uint64_t)));
  PIC_CUDA(cudaMalloc(&g.d_mlist_slot, PIC_MAX_SPECIES * cap * sizeof(int32_t)));
  g.mlist_cap = cap;
  return PIC_OK;
}


// Full-histogram selection of species s (used when the bounded selection
// does not apply or did not hold the ncoll smallest keys): histogram of all
// keys, the threshold bin found on the host, its candidates ordered on the
// host.  Leaves the ncoll selected slots in g.d_sel.
static int mcc_select_full(const MccK &k, int64_t ncoll, int64_t *misc_d) {
  if (int rc_ = zero_async(g.d_hist, 65536 * sizeof(uint32_t), g.st)) return rc_;
  if (int rc_ = zero_async(misc_d, kMccMisc * sizeof(int64_t), g.st)) return rc_;
  uint32_t *keys = g.d_sort_id;  // sort scratch, free while MCC runs
  k_mcc_hist<<<blocks_for(k.n, 256), 256, 0, g.st>>>(k, g.d_hist, keys);
  PIC_LAUNCHED();
  std::vector<uint32_t> hist(65536);
  PIC_CUDA(cudaMemcpyAsync(hist.data(), g.d_hist, 65536 * 4, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  int64_t below = 0;
  uint32_t bstar = 0;
  for (; bstar < 65536; ++bstar) {
    if (below + hist[bstar] >= ncoll) break;
    below += hist[bstar];
  }
  if (bstar >= 65536) {
    set_error("mcc: fewer live particles than collisions requested");
    return PIC_ERR_STATE;
  }
  const int64_t need = ncoll - below;
  const int64_t ncand_expect = hist[bstar];
  int rc = mcc_cand_alloc(ncand_expect + 4096);
  if (rc) return rc;
  k_mcc_pick<<<blocks_for(k.n, 256), 256, 0, g.st>>>(k, keys, bstar, g.d_sel, misc_d, g.d_cand, g.d_cand_slot,
                                                     g.cand_cap);
  PIC_LAUNCHED();
  int64_t misc[2];
  PIC_CUDA(cudaMemcpyAsync(misc, misc_d, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  const int64_t nsel = misc[0], ncand = misc[1];
  if (ncand != ncand_expect || nsel != below) {
    set_error("mcc: selection histogram mismatch");
    return PIC_ERR_CUDA;
  }
  std::vector<uint64_t> cand(ncand);
  std::vector<int32_t> cslot(ncand);
  PIC_CUDA(cudaMemcpy(cand.data(), g.d_cand, ncand * 8, cudaMemcpyDeviceToHost));
  PIC_CUDA(cudaMemcpy(cslot.data(), g.d_cand_slot, ncand * 4, cudaMemcpyDeviceToHost));
  std::vector<int64_t> order(ncand);
  for (int64_t i = 0; i < ncand; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cand[a] < cand[b]; });
  std::vector<int32_t> add(need);
  for (int64_t i = 0; i < need; ++i) add[i] = cslot[order[i]];
  if (need > 0) PIC_CUDA(cudaMemcpy(g.d_sel + nsel, add.data(), need * 4, cudaMemcpyHostToDevice));
  return PIC_OK;
}

// the bounded selection's sink of species s: key bound, list capacity,
// per-species histogram, list and counters
static MccSink mcc_sink(int s, uint64_t bound, int64_t lcap, uint32_t slo, uint32_t shi) {
  MccSink k;
  k.on = 1;
  k.rk = mcc_select_round_keys(slo, shi, (uint32_t)s, (uint32_t)g.P.seed, (uint32_t)(g.P.seed >> 32));
  k.bound = bound;
  k.id = g.sp[s].id;
  k.hist = g.d_hist + (size_t)s * 65536;
  k.lkey = g.d_mlist_key + (size_t)s * g.mlist_cap;
  k.lslot = g.d_mlist_slot + (size_t)s * g.mlist_cap;
  k.cap = lcap;
  k.cnt = reinterpret_cast<unsigned long long *>(g.d_msel + s * kMccSel);
  return k;
}

// the key bound that holds about `target` of n live keys (g.mcc_bound_scale
// < 1, a test hook, makes it too small, so the selection takes its fallback)
static uint64_t mcc_bound(double target, double n) {
  return std::max<uint64_t>(1, (uint64_t)std::ceil(g.mcc_bound_scale * target / n * 4294967296.0));
}

// about 2 ncoll + 64 keys below the bound, plus 8 standard deviations
static double mcc_target(double ncoll) { return 2.0 * ncoll + 64.0 + 8.0 * std::sqrt(2.0 * ncoll + 64.0); }

// Before the push of a step: the bounded selection of every species with
// MCC, sized for an upper bound of the step's ncoll (the push only removes
// particles), histograms and counters zeroed; the push fills them from the
// particles it leaves live (push_select) and mcc_run(prepared) goes on from
// there without reading the particles again.
int mcc_prepare(uint64_t step) {
  g.sel_step = ~0ull;
  const uint32_t slo = (uint32_t)step, shi = (uint32_t)(step >> 32);
  int64_t lcap[PIC_MAX_SPECIES] = {0}, lmax = 0;
  double target[PIC_MAX_SPECIES] = {0};
  for (int s = 0; s < g.ns; ++s) {
    g.sel_sink[s] = MccSink();
    g.sel_sink[s].on = 0;
    Species &sp = g.sp[s];
    if (!sp.has_mcc || sp.n_live == 0) continue;
    const int64_t nmax = (int64_t)((double)sp.n_live * sp.tab.collision_ratio) + 1;
    target[s] = mcc_target((double)nmax);
    if (g.mcc_full || target[s] >= 0.25 * (double)sp.n_live) continue;
    lcap[s] = (int64_t)(1.5 * target[s]) + 4096;
    lmax = std::max(lmax, lcap[s]);
  }
  if (lmax == 0) return PIC_OK;
  int rc;
  if ((rc = mcc_list_alloc(lmax))) return rc;
  for (int s = 0; s < g.ns; ++s) {
    if (lcap[s] == 0) continue;
    g.sel_sink[s] = mcc_sink(s, mcc_bound(target[s], (double)g.sp[s].n_live), lcap[s], slo, shi);
    if (int rc_ = zero_async(g.sel_sink[s].hist, 65536 * sizeof(uint32_t), g.st)) return rc_;
    if (int rc_ = zero_async(g.d_msel + s * kMccSel, kMccSel * sizeof(int64_t), g.st)) return rc_;
  }
  g.sel_step = step;
  return PIC_OK;
}

// MCC of every species with tables, one step.  Each species' selection and
// collisions are queued without waiting for the host: k_mcc_ties records
// whether the bounded selection holds the ncoll smallest keys and
// k_mcc_collide does nothing when it does not.  One read of the status
// blocks then finds the species (rarely any) that need the full selection;
// the created particles are ordered and appended on the device.
int mcc_run(uint64_t step, pic_mcc_stats *stats, bool prepared) {
  // the push of this step built the bounded selections (mcc_prepare)
  const bool prep = prepared && g.sel_step == step;
  g.sel_step = ~0ull;
  const uint32_t seed0 = (uint32_t)g.P.seed, seed1 = (uint32_t)(g.P.seed >> 32);
  const uint32_t slo = (uint32_t)step, shi = (uint32_t)(step >> 32);
  int64_t ncoll[PIC_MAX_SPECIES] = {0};
  bool bounded[PIC_MAX_SPECIES] = {false};
  int64_t most = 0;
  for (int s = 0; s < g.ns; ++s) {
    Species &sp = g.sp[s];
    if (!sp.has_mcc || sp.n_live == 0) continue;
    ncoll[s] = mcc_n_collisions(sp.n_live, sp.tab.collision_ratio, slo, shi, (uint32_t)s, seed0, seed1);
    if (stats) stats->n_selected[s] = ncoll[s];
    most = std::max(most, ncoll[s]);
  }
  if (most <= 0) return PIC_OK;
  // every buffer the queued kernels use is sized first: the bounded
  // selection's list for its largest species, the selection for the
  // largest ncoll
  int64_t lcap[PIC_MAX_SPECIES] = {0}, lmax = 0;
  for (int s = 0; s < g.ns; ++s) {
    if (ncoll[s] <= 0) continue;
    if (prep) {  // the prepared selections, whatever this step's ncoll
      bounded[s] = g.sel_sink[s].on != 0;
      continue;
    }
    const double npar = (double)g.sp[s].n_live;
    // the bound holds about 2 ncoll + 64 live keys (plus 8 standard
    // deviations); used while that is a small part of the species
    const double target = mcc_target((double)ncoll[s]);
    if (g.mcc_full || target >= 0.25 * npar) continue;
    bounded[s] = true;
    lcap[s] = (int64_t)(1.5 * target) + 4096;
    lmax = std::max(lmax, lcap[s]);
  }
  int rc;
  if ((rc = mcc_alloc(std::max<int64_t>(most, 1 << 16) + 4096))) return rc;
  if ((rc = mcc_cand_alloc(g.mcc_cap))) return rc;
  if ((rc = mcc_list_alloc(lmax))) return rc;  // no growth when prepared (lmax 0)
  if (int rc_ = zero_async(g.d_mcc_misc, PIC_MAX_SPECIES * kMccMisc * sizeof(int64_t), g.st)) return rc_;
  auto mk = [&](int s) {
    Species &sp = g.sp[s];
    return MccK{sp.x, sp.y, sp.vx, sp.vy, sp.vz, sp.loc, sp.id, sp.n_slots, seed0, seed1, slo, shi, (uint32_t)s,
                sp.f32 ? 1 : 0, mcc_select_round_keys(slo, shi, (uint32_t)s, seed0, seed1)};
  };
  auto collide = [&](int s, const int64_t *ok) -> int {
    Species &sp = g.sp[s];
    CollK c;
    c.k = mk(s);
    c.sel = g.d_sel;
    c.n_sel = ncoll[s];
    c.ok = ok;
    c.prob = sp.prob;
    c.tab = mc_table_from(sp.tab);
    c.gas.mass = g.gas.mass;
    c.gas.temperature = g.gas.temperature;
    c.mass = sp.mass;
    c.vref = g.v_ref;
    c.misc = g.d_mcc_misc + s * kMccMisc;
    c.ion_parent = g.d_ion_parent + s * g.mcc_cap;
    c.ion_data = g.d_ion_data + 6 * s * g.mcc_cap;
    c.ion_cap = g.mcc_cap;
    k_mcc_collide<<<blocks_for(ncoll[s], 128), 128, 0, g.st>>>(c);
    PIC_LAUNCHED();
    return PIC_OK;
  };
  // 1. bounded selections and their collisions, queued
  for (int s = 0; s < g.ns; ++s) {
    if (!bounded[s]) continue;
    int64_t *ms = g.d_msel + s * kMccSel, *misc = g.d_mcc_misc + s * kMccMisc;
    MccSink sink;
    if (prep) {
      sink = g.sel_sink[s];
    } else {
      sink = mcc_sink(s, mcc_bound(mcc_target((double)ncoll[s]), (double)g.sp[s].n_live), lcap[s], slo, shi);
      if (int rc_ = zero_async(sink.hist, 65536 * sizeof(uint32_t), g.st)) return rc_;
      if (int rc_ = zero_async(ms, kMccSel * sizeof(int64_t), g.st)) return rc_;
      const MccK k = mk(s);
      k_mcc_scan<<<blocks_for((k.n + 3) / 4, 256), 256, 0, g.st>>>(k, sink);
      PIC_LAUNCHED();
    }
    k_mcc_bstar<<<1, 1024, 0, g.st>>>(sink.hist, ncoll[s], ms);
    PIC_LAUNCHED();
    k_mcc_pick_list<<<(unsigned)std::min<int64_t>(blocks_for(sink.cap, 256), 1184), 256, 0, g.st>>>(
        sink.lkey, sink.lslot, sink.cnt, sink.cap, sink.bound, ms, g.d_sel, g.d_cand, g.d_cand_slot, g.cand_cap,
        misc);
    PIC_LAUNCHED();
    k_mcc_ties<<<1, 1024, 0, g.st>>>(g.d_cand, g.d_cand_slot, g.cand_cap, sink.cap, ms, misc, ncoll[s], g.d_sel);
    PIC_LAUNCHED();
    if ((rc = collide(s, ms + 4))) return rc;
  }
  // 2. one read of every status block; full selections where needed
  int64_t ms_h[PIC_MAX_SPECIES * kMccSel], misc_h[PIC_MAX_SPECIES * kMccMisc];
  PIC_CUDA(cudaMemcpyAsync(ms_h, g.d_msel, sizeof ms_h, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaMemcpyAsync(misc_h, g.d_mcc_misc, sizeof misc_h, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  for (int s = 0; s < g.ns; ++s) {
    if (ncoll[s] <= 0 || (bounded[s] && ms_h[s * kMccSel + 4] == 1)) continue;
    int64_t *misc = g.d_mcc_misc + s * kMccMisc;
    if ((rc = mcc_select_full(mk(s), ncoll[s], misc))) return rc;
    if ((rc = collide(s, nullptr))) return rc;
    PIC_CUDA(cudaMemcpyAsync(misc_h + s * kMccMisc, misc, kMccMisc * sizeof(int64_t), cudaMemcpyDeviceToHost,
                             g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
  }
  // 3. ionisations: the host reads only the counts; each species' are put in
  // parent-id order and appended on the device (MCCAddNewParticle, after
  // every species collided)
  int64_t nion[PIC_MAX_SPECIES] = {0};
  for (int s = 0; s < g.ns; ++s) {
    if (ncoll[s] <= 0) continue;
    const int64_t *m2 = misc_h + s * kMccMisc;
    if (stats)
      for (int r = 0; r < g.sp[s].tab.n_reaction && r < 8; ++r) stats->n_by_reaction[s][r] = m2[2 + r];
    nion[s] = m2[12];
    if (nion[s] > g.mcc_cap) {
      set_error("mcc: ionisation buffer overflow");
      return PIC_ERR_CAPACITY;
    }
  }
  for (int s = 0; s < g.ns; ++s) {
    const int64_t n = nion[s];
    if (n == 0) continue;
    if (n > g.mcc_new_cap) {  // grow the created-particle buffers (kept across steps)
      PIC_CUDA(cudaStreamSynchronize(g.st));
      cudaFree(g.d_mcc_pslot);
      cudaFree(g.d_mcc_vel);
      cudaFree(g.d_ion_order);
      g.d_mcc_pslot = nullptr;
      g.d_mcc_vel = nullptr;
      g.d_ion_order = nullptr;
      g.mcc_new_cap = 0;
      const int64_t cap = std::max<int64_t>(2 * n, 1 << 16);
      PIC_CUDA(cudaMalloc(&g.d_mcc_pslot, cap * 4));
      PIC_CUDA(cudaMalloc(&g.d_mcc_vel, 6 * cap * 8));
      PIC_CUDA(cudaMalloc(&g.d_ion_order, cap * 4));
      g.mcc_new_cap = cap;
    }
    const int64_t *parent = g.d_ion_parent + s * g.mcc_cap;
    double *vel_e = g.d_mcc_vel, *vel_i = g.d_mcc_vel + 3 * g.mcc_new_cap;
    k_ion_rank<<<blocks_for(n, 128), 128, 0, g.st>>>(parent, n, g.d_ion_order);
    PIC_LAUNCHED();
    k_ion_build<<<blocks_for(n, 256), 256, 0, g.st>>>(parent, g.d_ion_data + 6 * s * g.mcc_cap, g.d_ion_order, n,
                                                      g.v_ref, g.d_mcc_pslot, vel_e, vel_i);
    PIC_LAUNCHED();
    // the created electron joins species s; the ion the ionisation
    // reaction's resultant
    int ion_species = -1;
    for (int r = 0; r < g.sp[s].tab.n_reaction; ++r)
      if (g.sp[s].tab.reaction_type[r] == 13) ion_species = g.sp[s].tab.resultant[r];
    Species &from = g.sp[s];
    for (int which = 0; which < 2; ++which) {
      const int ts = which == 0 ? s : ion_species;
      if (ts < 0 || ts >= g.ns) continue;
      Species &to = g.sp[ts];
      if (to.n_slots + n > to.capacity) {
        set_error("mcc: particle capacity exceeded by ionisation");
        return PIC_ERR_CAPACITY;
      }
      AppendK a{from.x, from.y, from.loc, to.x, to.y, to.vx, to.vy, to.vz, to.loc, to.id,
                to.n_slots, to.next_id, g.d_mcc_pslot, which == 0 ? vel_e : vel_i, n, to.f32 ? 1 : 0};
      k_mcc_append<<<blocks_for(n, 256), 256, 0, g.st>>>(a);
      PIC_LAUNCHED();
      to.n_slots += n;
      to.n_live += n;
      to.next_id += (uint32_t)n;
      if (stats) stats->n_created[ts] += n;
    }
  }
  return PIC_OK;
}

}  // namespace pic

using namespace pic;

extern "C" int pic_mcc_init(const pic_gas *gas, int32_t n_tables, const pic_mcc_table *tables) {
  if (!g.inited) {
    set_error("pic_mcc_init: library not initialised");
    return PIC_ERR_STATE;
  }
  if (!gas || n_tables < 0 || (n_tables > 0 && !tables)) {
    set_error("pic_mcc_init: bad arguments");
    return PIC_ERR_ARG;
  }
  g.gas = *gas;
  for (int t = 0; t < n_tables; ++t) {
    const pic_mcc_table &T = tables[t];
    if (T.species < 0 || T.species >= g.ns || T.n_reaction < 1 || T.n_reaction > PIC_MAX_REACTIONS ||
        T.n_sigma < 2 || !T.probability || !(T.collision_ratio >= 0 && T.collision_ratio < 1)) {
      set_error("pic_mcc_init: bad table");
      return PIC_ERR_ARG;
    }
    Species &sp = g.sp[T.species];
    sp.tab = T;
    sp.has_mcc = true;
    if (sp.prob) cudaFree(sp.prob);
    size_t n = (size_t)T.n_sigma * T.n_reaction;
    PIC_CUDA(cudaMalloc(&sp.prob, n * sizeof(double)));
    PIC_CUDA(cudaMemcpy(sp.prob, T.probability, n * sizeof(double), cudaMemcpyHostToDevice));
    sp.tab.probability = nullptr;
  }
  if (!g.d_hist) PIC_CUDA(cudaMalloc(&g.d_hist, PIC_MAX_SPECIES * 65536 * sizeof(uint32_t)));
  if (!g.d_mcc_misc) PIC_CUDA(cudaMalloc(&g.d_mcc_misc, PIC_MAX_SPECIES * kMccMisc * sizeof(int64_t)));
  g.mcc_ready = n_tables > 0;
  return PIC_OK;
}

extern "C" int pic_mcc(uint64_t step, pic_mcc_stats *stats) {
  if (!g.inited) {
    set_error("pic_mcc: library not initialised");
    return PIC_ERR_STATE;
  }
  pic_mcc_stats local;
  std::memset(&local, 0, sizeof local);
  int rc = g.mcc_ready ? mcc_run(step, &local) : PIC_OK;
  if (stats) *stats = local;
  return rc;
}
