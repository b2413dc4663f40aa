// picgpu.cu -- B200 kernels and C-ABI of the IFE-PIC step.
//
// Layout in HBM
//   particles : SoA per species, FP64 x, y, vx, vy, vz, int32 element (loc),
//               uint32 id; loc = -1 marks an absorbed slot until the next sort.
//   fields    : node-indexed FP64 arrays on the full nnx*nny grid
//               (n = i*nny + j); Dirichlet nodes hold 0 in the PCG vectors.
//   deposit   : int64 fixed-point accumulators per species and node.
//
// Kernels (all FP64; compiled with --fmad=false, FMAs are written explicitly
// so the CPU oracle repeats the same roundings):
//   k_locate ........ InjectPositioning.f90:1-24 / GetParChg_2D.f90:137-163
//   k_push .......... MoveOne.f90 + Get_ParticleEField_PPR.f90 +
//                     AdjustParticleBoundary (MCCInterface.f90:361-532), fused
//                     with locate + bilinear deposit (GetParChg_2D.f90:788-843)
//   k_rho ........... GetParChg_2D.f90:849-911 (normalise by dual volume)
//   k_rhs ........... Global_RHS_PDE_2D.f90:72-138 + IFE_Solve_2D.f90:188-192
//   k_pcg_* ......... MY_PCG.f90:56-127 with MATVEC_1/MSOLVE_1
//   k_ppr ........... GetEfield_SIDG_PPR.f90:153-304
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pic_ctx.h"

namespace pic {

Ctx g;
long long g_launches = 0;
static std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
int cuda_fail(cudaError_t e, const char *where) {
  g_err = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  return PIC_ERR_CUDA;
}

// ----------------------------------------------------------------------------
// device helpers
// ----------------------------------------------------------------------------

struct FieldK {
  const double *efx, *efy;
  const double *c2, *c3, *c4, *c5, *c6;
  const double2 *efxy;  // {efx, efy} per node: the gather's four nodes in four 16-byte loads
};

// ci, cj: the element's column and row (0-based), set when it is found
__device__ __forceinline__ int locate_elem(const MeshK &m, double x, double y, int &ci, int &cj) {
  // InjectPositioning.f90:13-22: i = INT((x - dxmin)/dx) + 1 (1-based)
  double rxp = (x - m.xmin) / m.hx;
  double ryp = (y - m.ymin) / m.hy;
  int i = (int)rxp + 1;
  int j = (int)ryp + 1;
  if (i == m.nnx) i = m.nnx - 1;  // GetParChg_2D.f90:143-149 clamp
  if (j == m.nny) j = m.nny - 1;
  if (!(rxp >= 0.0) || !(ryp >= 0.0) || i < 1 || j < 1 || i > m.nex || j > m.ney) return -1;
  ci = i - 1;
  cj = j - 1;
  return (i - 1) * m.ney + (j - 1);
}

__device__ __forceinline__ int locate_elem(const MeshK &m, double x, double y) {
  int ci, cj;
  return locate_elem(m, x, y, ci, cj);
}

// e / ney without a division: with M = floor(2^32 / ney) + 1, umulhi(e, M)
// exceeds e / ney by less than e / 2^32 < 1, so it is the quotient or one
// more, and one correction makes it exact for every element id (ney >= 2).
__device__ __forceinline__ int elem_column(const MeshK &m, int e) {
  int i = (int)__umulhi((unsigned)e, m.ney_magic);
  if (i * m.ney > e) --i;
  return i;
}

// The element's node coordinates are computed, not loaded: xs[i] is
// xmin + hx*i (one product and one sum, correctly rounded on the host and,
// without contraction, here), so the values are the same bits.
__device__ __forceinline__ double node_x(const MeshK &m, int i) { return m.xmin + m.hx * (double)i; }
__device__ __forceinline__ double node_y(const MeshK &m, int j) { return m.ymin + m.hy * (double)j; }

// bilinear weights and nodes of the element in column i, row j
__device__ __forceinline__ void bilinear_ij(const MeshK &m, int i, int j, double x, double y, double W[4],
                                            int nodes[4]) {
  double x1 = node_x(m, i), x2 = node_x(m, i + 1), y1 = node_y(m, j), y2 = node_y(m, j + 1);
  double hxp = x2 - x1, hyp = y2 - y1;
  double dx = (x - x1) / hxp;
  double dy = (y - y1) / hyp;
  double xc = 1.0 - dx, yc = 1.0 - dy;
  W[0] = xc * yc;
  W[1] = dx * yc;
  W[2] = dx * dy;
  W[3] = xc * dy;
  int n1 = i * m.nny + j;
  nodes[0] = n1;
  nodes[1] = n1 + m.nny;
  nodes[2] = n1 + m.nny + 1;
  nodes[3] = n1 + 1;
}

__device__ __forceinline__ void bilinear(const MeshK &m, int e, double x, double y, double W[4],
                                         int nodes[4], int *ie, int *je) {
  int i = elem_column(m, e), j = e - i * m.ney;
  bilinear_ij(m, i, j, x, y, W, nodes);
  *ie = i;
  *je = j;
}

// Canonical block reduction of up to 3 values (see PIC_RED_* in pic_common.h).
template <int NV>
__device__ __forceinline__ void block_sum_canon(double v[NV], double *out /*[NV], thread 0*/) {
  __shared__ double ws[NV][PIC_RED_THREADS / 32];
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int off = 16; off > 0; off >>= 1) v[k] = v[k] + __shfl_xor_sync(0xffffffffu, v[k], off);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int k = 0; k < NV; ++k) ws[k][w] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int q = 0; q < PIC_RED_THREADS / 32; ++q) s = s + ws[k][q];
      out[k] = s;
    }
  __syncthreads();
}

// Final reduction of nb per-block partials by the last block (canonical order).
template <int NV>
__device__ __forceinline__ void final_sum_canon(const double *part, int nb, double *out) {
  double v[NV];
  for (int k = 0; k < NV; ++k) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += PIC_RED_THREADS) a = a + __ldcg(part + (size_t)k * nb + b);
    v[k] = a;
  }
  block_sum_canon<NV>(v, out);
}

__device__ __forceinline__ bool arrive_last(unsigned int *ticket) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return last;
}

// ----------------------------------------------------------------------------
// particle kernels
// ----------------------------------------------------------------------------

__global__ void k_locate(MeshK m, const double *__restrict__ x, const double *__restrict__ y,
                         int32_t *__restrict__ loc, int64_t begin, int64_t end,
                         unsigned long long *bad) {
  int64_t p = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= end) return;
  if (loc[p] < 0 && loc[p] != -2) return;  // absorbed slot stays absorbed
  int e = locate_elem(m, x[p], y[p]);
  if (e < 0) atomicAdd(bad, 1ull);
  loc[p] = e;
}

struct PushK {
  double qm, dt, mass, vref;
  int do_push, do_deposit, do_energy;
  int wall[4];
};

struct SpK {
  double *x, *y, *vx, *vy, *vz;
  int32_t *loc;
  unsigned long long *q_acc, *e_acc;
  unsigned long long *lost, *bad;
  int64_t n;
  unsigned long long *fail;  // a bounded wait of the bulk-staged push ran out
  MccSink sel;               // the step's MCC selection, built from the particles left live
};

__constant__ ObjK c_obj;

__device__ __forceinline__ bool absorbed_by_object(double x, double y) {
  for (int k = 0; k < c_obj.n; ++k) {
    const pic_object &o = c_obj.o[k];
    if (o.shape == PIC_SHAPE_CIRCLE) {
      double dx = x - o.cx, dy = y - o.cy;
      if (dx * dx + dy * dy < o.a * o.a) return true;
    } else if (o.shape == PIC_SHAPE_BOX) {
      if (x > o.cx && x < o.a && y > o.cy && y < o.b) return true;
    } else if (o.shape == PIC_SHAPE_ELLIPSE) {
      // outside the box of half-width max(a, b): outside the ellipse
      if (fabs(x - o.cx) > c_obj.half[k] || fabs(y - o.cy) > c_obj.half[k]) continue;
      const double c = c_obj.ca[k], s = c_obj.sa[k];
      double u = (x - o.cx) * c + (y - o.cy) * s;
      double v = -(x - o.cx) * s + (y - o.cy) * c;
      if ((u * u) / (o.a * o.a) + (v * v) / (o.b * o.b) < 1.0) return true;
    }
  }
  return false;
}

// Segmented warp sums of N int64 values over lanes [lane, seg_end] of one
// segment (reduction toward the segment head).  After the steps off = 1, 2,
// .., 2^(k-1) lane i holds the sum over [i, min(i + 2^k - 1, seg_end)], so
// the steps stop once off reaches the warp's longest run `maxlen` (the same
// for every lane): a warp of runs of at most 8 takes 3 steps instead of 5.
constexpr double kNarrowScale = 16777216.0;  // 2^24: the mixed-precision charge's unit
constexpr int kNarrowShift = 16;             // 2^24 -> 2^40 (PIC_Q_SCALE)

template <int N>
__device__ __forceinline__ void seg_sums(long long (&v)[N], int lane, int seg_end, int maxlen) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    if (off >= maxlen) break;
    const bool take = lane + off <= seg_end;
#pragma unroll
    for (int c = 0; c < N; ++c) {
      const long long o = __shfl_down_sync(0xffffffffu, v[c], off);
      if (take) v[c] += o;
    }
  }
}

// The same over 32-bit values (the mixed-precision charge, below).
template <int N>
__device__ __forceinline__ void seg_sums32(unsigned (&v)[N], int lane, int seg_end, int maxlen) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    if (off >= maxlen) break;
    const bool take = lane + off <= seg_end;
#pragma unroll
    for (int c = 0; c < N; ++c) {
      const unsigned o = __shfl_down_sync(0xffffffffu, v[c], off);
      if (take) v[c] += o;
    }
  }
}

// Lost-particle count and fixed-point deposit of one warp's particles (key =
// the particle's element, -1 for none).  Segmented warp aggregation by
// element (particles are cell-sorted, so neighbouring lanes usually share an
// element), then one atomic per node and value from the segment head.
// Integer sums are exact: node totals do not depend on the segmentation.
// CONSERVE (Cartesian meshes, FP64 and mixed precision): corner 2's charge
// is 2^40 minus the other three rounded corners, so every particle deposits
// exactly 2^40 and a run of L particles 2^40 L minus three sums -- one 64-bit
// warp sum fewer (the oracle rounds the same way).  Without it (the r-z
// weights, which do not sum to 1 on the axis row) each corner is rounded on
// its own.
// NARROW (mixed precision, Cartesian, with CONSERVE): the three corners are
// rounded to 2^-24 of a particle -- the resolution of the FP32 offsets they
// come from -- so a warp's sums fit in 32 bits (32 x 2^24 < 2^30): one
// shuffle and one add a value and step instead of two each; the head scales
// them to the accumulator's 2^-40 units, and corner 2 keeps every particle's
// charge exactly 2^40.  The energy deposit stays 64-bit.
template <bool CONSERVE = false, bool NARROW = false>
__device__ __forceinline__ void warp_deposit(const SpK &s, int lane, int key, const double W[4], const int nodes[4],
                                             double energy, bool lost, int do_deposit, int do_energy) {
  unsigned int lm = __ballot_sync(0xffffffffu, lost);
  if (lane == 0 && lm) atomicAdd(s.lost, (unsigned long long)__popc(lm));
  if (!do_deposit) return;
  const int key0 = __shfl_sync(0xffffffffu, key, 0);  // every lane, before any test
  if (__all_sync(0xffffffffu, key >= 0 && key == key0)) {
    // one element for the whole warp: exact integer warp sums with redux on
    // the low 24 bits and the rest (values are non-negative; the sums fit in
    // 32 bits for values below 2^51, i.e. particle energies below ~5e5 eV)
    auto wsum = [&](long long v) {
      const unsigned lo = (unsigned)(v & 0xffffff), hi = (unsigned)(v >> 24);
      return ((long long)__reduce_add_sync(0xffffffffu, hi) << 24) + (long long)__reduce_add_sync(0xffffffffu, lo);
    };
    long long qv[4];
    if (NARROW) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c != 2)
          qv[c] = (long long)__reduce_add_sync(0xffffffffu, (unsigned)__double2uint_rn(W[c] * kNarrowScale))
                  << kNarrowShift;
    } else {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (!CONSERVE || c != 2) qv[c] = wsum(__double2ll_rn(W[c] * PIC_Q_SCALE));
    }
    if (CONSERVE) qv[2] = 32ll * (1ll << 40) - ((qv[0] + qv[1]) + qv[3]);
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < 4; ++c) atomicAdd(s.q_acc + nodes[c], (unsigned long long)qv[c]);
    if (!do_energy) return;
#pragma unroll
    for (int c = 0; c < 4; ++c) qv[c] = wsum(__double2ll_rn((W[c] * energy) * PIC_E_SCALE));
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < 4; ++c) atomicAdd(s.e_acc + nodes[c], (unsigned long long)qv[c]);
    return;
  }
  int prev = __shfl_up_sync(0xffffffffu, key, 1);
  bool head = (lane == 0) || (key != prev);
  unsigned int heads = __ballot_sync(0xffffffffu, head);
  unsigned int above = (lane == 31) ? 0u : (heads & ~((2u << lane) - 1u));
  int seg_end = above ? (__ffs(above) - 2) : 31;
  const int maxlen = (int)__reduce_max_sync(0xffffffffu, head ? (unsigned)(seg_end - lane + 1) : 0u);
  long long qv[4];
  if (NARROW) {
    unsigned q3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) q3[c] = (key >= 0) ? __double2uint_rn(W[c == 2 ? 3 : c] * kNarrowScale) : 0u;
    seg_sums32(q3, lane, seg_end, maxlen);
    qv[0] = (long long)q3[0] << kNarrowShift;
    qv[1] = (long long)q3[1] << kNarrowShift;
    qv[3] = (long long)q3[2] << kNarrowShift;
    qv[2] = (long long)(seg_end - lane + 1) * (1ll << 40) - ((qv[0] + qv[1]) + qv[3]);
  } else if (CONSERVE) {
    long long q3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) q3[c] = (key >= 0) ? __double2ll_rn(W[c == 2 ? 3 : c] * PIC_Q_SCALE) : 0ll;
    seg_sums(q3, lane, seg_end, maxlen);
    // the head's sums cover its run, lanes [lane, seg_end]
    qv[0] = q3[0];
    qv[1] = q3[1];
    qv[3] = q3[2];
    qv[2] = (long long)(seg_end - lane + 1) * (1ll << 40) - ((qv[0] + qv[1]) + qv[3]);
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) qv[c] = (key >= 0) ? __double2ll_rn(W[c] * PIC_Q_SCALE) : 0ll;
    seg_sums(qv, lane, seg_end, maxlen);
  }
  if (head && key >= 0)
#pragma unroll
    for (int c = 0; c < 4; ++c) atomicAdd(s.q_acc + nodes[c], (unsigned long long)qv[c]);
  if (!do_energy) return;
  long long ev[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) ev[c] = (key >= 0) ? __double2ll_rn((W[c] * energy) * PIC_E_SCALE) : 0ll;
  seg_sums(ev, lane, seg_end, maxlen);
  if (head && key >= 0)
#pragma unroll
    for (int c = 0; c < 4; ++c) atomicAdd(s.e_acc + nodes[c], (unsigned long long)ev[c]);
}

// The MCC selection of the step (the bounded one of the MCC pass, same
// keys, same histogram and list) from the particles this push leaves live
// (key >= 0: deposited), so the MCC pass does not read the particles again.
// Every lane takes part.  The id is loaded at the start of the particle's
// work (push_select_id), so its latency hides behind the push.
__device__ __forceinline__ uint32_t push_select_id(const SpK &s, int64_t p) {
  return s.sel.on && p < s.n ? __ldcs(s.sel.id + p) : 0u;
}

__device__ __forceinline__ void push_select(const SpK &s, int lane, int key, int64_t p, uint32_t id) {
  if (!s.sel.on) return;  // the same for every lane
  uint32_t k = 0;
  bool want = false;
  if (key >= 0) {
    k = mcc_select_key(id, s.sel.rk);
    want = (uint64_t)k < s.sel.bound;
  }
  mcc_sink_put(s.sel, lane, want, k, id, p);
}

// The same for the persistent bulk-staged pushes, without a global atomic
// that a warp waits on inside the tile loop: entries go to a per-CTA
// shared-memory buffer (a shared atomic each) and reach the global list in
// one reservation when the CTA ends; past kSelBuf entries they go straight
// to the global list.  Only lanes with a selected particle do anything.
constexpr int kSelBuf = 256;
struct SelBuf {
  uint64_t key[kSelBuf];
  int32_t slot[kSelBuf];
  int n;
  unsigned long long base;
};

__device__ __forceinline__ void push_select_cta(const SpK &s, int key, int64_t p, uint32_t id, SelBuf &b) {
  if (!s.sel.on || key < 0) return;
  const uint32_t k = mcc_select_key(id, s.sel.rk);
  if ((uint64_t)k >= s.sel.bound) return;
  atomicAdd(s.sel.hist + mcc_bin(k, s.sel.bound), 1u);
  const uint64_t kv = ((uint64_t)k << 32) | (uint64_t)id;
  const int i = atomicAdd(&b.n, 1);
  if (i < kSelBuf) {
    b.key[i] = kv;
    b.slot[i] = (int32_t)p;
  } else {
    const unsigned long long j = atomicAdd(s.sel.cnt, 1ull);
    if (j < (unsigned long long)s.sel.cap) {
      s.sel.lkey[j] = kv;
      s.sel.lslot[j] = (int32_t)p;
    }
  }
}

// every thread of the CTA, after its last tile
__device__ __forceinline__ void push_select_flush(const SpK &s, SelBuf &b) {
  if (!s.sel.on) return;  // the same for every thread
  __syncthreads();
  const int n = min(b.n, kSelBuf);
  if (threadIdx.x == 0) b.base = n > 0 ? atomicAdd(s.sel.cnt, (unsigned long long)n) : 0ull;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned long long j = b.base + (unsigned long long)i;
    if (j < (unsigned long long)s.sel.cap) {
      s.sel.lkey[j] = b.key[i];
      s.sel.lslot[j] = b.slot[i];
    }
  }
}

// Axisymmetric deposit weights (delta = 1, r = y), GetParChg_2D.f90:803-821:
// linear in r^2 across the element, the two lower nodes scaled by 0.75 in
// the element row on the axis; R1 = ymin + y1 and R2 = ymin + y2 as there.
__device__ __forceinline__ void weights_axi(const MeshK &m, int e, double x, double y, double W[4],
                                            int nodes[4]) {
  int i = elem_column(m, e), j = e - i * m.ney;
  double x1 = node_x(m, i), x2 = node_x(m, i + 1), y1 = node_y(m, j), y2 = node_y(m, j + 1);
  double dx = (x - x1) / (x2 - x1), xc = 1.0 - dx;
  double beta = (fabs(y1 - m.ymin) < 1e-5) ? 0.75 : 1.0;
  double R1 = m.ymin + y1, R2 = m.ymin + y2;
  double den = R2 * R2 - R1 * R1;
  W[0] = ((xc * (R2 * R2 - y * y)) / den) * beta;
  W[1] = ((dx * (R2 * R2 - y * y)) / den) * beta;
  W[2] = (dx * (y * y - R1 * R1)) / den;
  W[3] = (xc * (y * y - R1 * R1)) / den;
  int n1 = i * m.nny + j;
  nodes[0] = n1;
  nodes[1] = n1 + m.nny;
  nodes[2] = n1 + m.nny + 1;
  nodes[3] = n1 + 1;
}

// One live FP64 particle p (element e, position and velocity as loaded):
// gather E (old element), leapfrog push, wall/object absorption, locate;
// writes the particle back and returns what the warp deposit needs.
// AXI (delta = 1, MoveOne.f90:213-263): x = z, y = r and the velocity held in
// the particle's own frame (vx = v_z, vy = v_r, vz = v_theta); after the kick
// the transverse move X = r + dt v_r, Y = dt v_theta gives r' = |(X, Y)| and
// (v_r, v_theta) is rotated into the new frame by (X, Y)/r'; the deposit
// weights are weights_axi.
template <bool AXI>
__device__ __forceinline__ void push_fp64_one(const MeshK &m, const FieldK &f, const PushK &prm, const SpK &s,
                                              int64_t p, int e, double x, double y, double vx, double vy,
                                              int &key, double W[4], int nodes[4], double &energy, bool &lost) {
  int en = -2;          // the new element, once located
  int ci = 0, cj = 0;   // and its column and row
  if (prm.do_push) {
    int ie, je;
    bilinear(m, e, x, y, W, nodes, &ie, &je);
    double Ex, Ey;
    if (m.element_index[e] > 0) {
      // Get_ParticleEField_PPR.f90:19-33: average of the PPR gradients of the
      // element's outside nodes
      double ex = 0.0, ey = 0.0;
      int cnt = 0;
      for (int c = 0; c < 4; ++c) {
        int n = nodes[c];
        if (m.node_index[n] == -1) {
          ++cnt;
          int ni = n / m.nny, nj = n - ni * m.nny;
          double xr = x - m.xs[ni], yr = y - m.ys[nj];
          ex = ((ex + f.c2[n]) + (2.0 * f.c4[n]) * xr) + f.c5[n] * yr;
          ey = ((ey + f.c3[n]) + (2.0 * f.c6[n]) * yr) + f.c5[n] * xr;
        }
      }
      ex = ex / (double)cnt;
      ey = ey / (double)cnt;
      Ex = -ex;
      Ey = -ey;
    } else {
      const double2 e0 = f.efxy[nodes[0]], e1 = f.efxy[nodes[1]], e2 = f.efxy[nodes[2]], e3 = f.efxy[nodes[3]];
      Ex = ((W[0] * e0.x + W[1] * e1.x) + W[2] * e2.x) + W[3] * e3.x;
      Ey = ((W[0] * e0.y + W[1] * e1.y) + W[2] * e2.y) + W[3] * e3.y;
    }
    vx = vx + (prm.qm * Ex) * prm.dt;
    vy = vy + (prm.qm * Ey) * prm.dt;
    if (AXI) {
      double vt = s.vz[p];
      double X = y + prm.dt * vy, Y = prm.dt * vt;
      if (X == 0.0) X = m.hy * (double)1.0e-5f;
      const double rn = sqrt(X * X + Y * Y), c = X / rn, sn = Y / rn;
      const double vr = c * vy + sn * vt;
      vt = c * vt - sn * vy;
      vy = vr;
      s.vz[p] = vt;
      x = x + prm.dt * vx;
      y = rn;
    } else {
      x = x + prm.dt * vx;
      y = y + prm.dt * vy;
    }
    // walls: left, right, bottom (not the axis), top
    if (x <= m.xmin) {
      if (prm.wall[0] == PIC_WALL_REFLECT) { x = m.xmin + (m.xmin - x); vx = -vx; }
      else lost = true;
    } else if (x > m.xmax) {
      if (prm.wall[1] == PIC_WALL_REFLECT) { x = m.xmax - (x - m.xmax); vx = -vx; }
      else lost = true;
    } else if (!AXI && y < m.ymin) {
      if (prm.wall[2] == PIC_WALL_REFLECT) { y = m.ymin + (m.ymin - y); vy = -vy; }
      else lost = true;
    } else if (y > m.ymax) {
      if (prm.wall[3] == PIC_WALL_REFLECT) { y = m.ymax - (y - m.ymax); vy = -vy; }
      else lost = true;
    }
    // objects: only a particle in an element whose box meets an object's
    // bounding box (a flag built at init, with a cell of margin) can be
    // inside one, so the exact test runs there only
    if (!lost) {
      en = locate_elem(m, x, y, ci, cj);
      if ((en < 0 || m.elem_near[en]) && absorbed_by_object(x, y)) lost = true;
    }
    s.x[p] = x;
    s.y[p] = y;
    s.vx[p] = vx;
    s.vy[p] = vy;
  }
  if (lost) {
    s.loc[p] = -1;
  } else if (prm.do_deposit) {
    if (en == -2) en = locate_elem(m, x, y, ci, cj);
    if (en < 0) {
      atomicAdd(s.bad, 1ull);
      s.loc[p] = -1;
      lost = true;
    } else {
      s.loc[p] = en;
      key = en;
      if (AXI) {
        weights_axi(m, en, x, y, W, nodes);
      } else {
        bilinear_ij(m, ci, cj, x, y, W, nodes);
      }
      if (prm.do_energy) {  // the per-node energy is deposited on diagnostic steps only
        const double vz = s.vz[p];
        energy = ((((0.5 * prm.mass) * ((vx * vx + vy * vy) + vz * vz)) * prm.vref) * prm.vref) /
                 PIC_JTOEV;
      }
    }
  }
}

// One particle per thread, loaded directly: push_fp64_one, then the warp's
// fixed-point deposit of weight and weight*energy.
template <bool AXI>
__global__ void __launch_bounds__(256, 4) k_push(MeshK m, FieldK f, PushK prm, SpK s) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
  int lane = threadIdx.x & 31;
  int key = -1;
  double W[4] = {0, 0, 0, 0};
  int nodes[4] = {0, 0, 0, 0};
  double energy = 0.0;
  bool lost = false;
  if (p < s.n) {
    int e = s.loc[p];
    if (e >= 0) push_fp64_one<AXI>(m, f, prm, s, p, e, s.x[p], s.y[p], s.vx[p], s.vy[p], key, W, nodes, energy, lost);
  }
  warp_deposit<!AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
  push_select(s, lane, key, p, pid);
}

struct PushM {
  float qmdt;      // q/m * dt
  float dtx, dty;  // dt/hx, dt/hy: cells moved per unit velocity per step
  float hx, hy;
  double dt, hyd, inv_hy;  // the r-z move (FP64): dt, hy and 1/hy
  double mass, vref;
  int do_push, do_deposit, do_energy;
  int wall[4];
};

// Mixed-precision form of k_push (PIC_PREC_MIXED): the particle is its
// element (int32) plus FP32 offsets inside it (element widths) and FP32
// velocities; the gather reads 32-byte FP32 node records {efx, efy, c2..c6},
// the move is in element units (no division), walls are decided on (element,
// offset) exactly, the object test runs in FP64 on the absolute position, and
// the deposit is the same int64 fixed point.  40 bytes per particle (44 with
// vz on diagnostic steps) against 80 for k_push.
// push_mixed_one: one live particle p (element e, offsets ax, ay,
// velocities vx, vy as loaded): gather, push, walls, objects, locate; writes
// the particle back and returns what the warp deposit needs.
// AXI (r-z, y = r with the axis at ymin = 0; vx, vy, vz = v_z, v_r, v_theta
// in the particle's frame): the axial move as above; the transverse move, as
// k_push<true> does it, in FP64 from the absolute radius r = (j + ay) hy --
// X = r + dt v_r, Y = dt v_theta, r' = |(X, Y)|, (v_r, v_theta) rotated by
// (X, Y)/r' -- and r' split back into (j, ay); the deposit weights are
// k_push<true>'s r^2-linear ones written in the offsets:
// (1 - a)(2j + 1 + a)/(2j + 1) below, a(2j + a)/(2j + 1) above, x 0.75 below
// in the axis row.
template <bool AXI>
__device__ __forceinline__ void push_mixed_one(const MeshK &m, const float *__restrict__ c32, const PushM &prm,
                                               const SpK &s, int64_t p, int e, float ax, float ay, float vx,
                                               float vy, int &key, double W[4], int nodes[4], double &energy,
                                               bool &lost) {
  float *fx = reinterpret_cast<float *>(s.x), *fy = reinterpret_cast<float *>(s.y);
  float *fvx = reinterpret_cast<float *>(s.vx), *fvy = reinterpret_cast<float *>(s.vy);
  float *fvz = reinterpret_cast<float *>(s.vz);
  int i = elem_column(m, e), j = e - i * m.ney;
  float vt = 0.f;  // AXI: v_theta after the push
  if (prm.do_push) {
    const int n1 = i * m.nny + j;
    const int cn[4] = {n1, n1 + m.nny, n1 + m.nny + 1, n1 + 1};
    float Ex, Ey;
    if (m.element_index[e] > 0) {
      // average of the PPR gradients of the element's outside nodes
      const float ox[4] = {0.f, 1.f, 1.f, 0.f}, oy[4] = {0.f, 0.f, 1.f, 1.f};
      float ex = 0.f, ey = 0.f;
      int cnt = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (m.node_index[cn[c]] != -1) continue;
        ++cnt;
        const float4 r0 = *reinterpret_cast<const float4 *>(c32 + 8 * (size_t)cn[c]);
        const float4 r1 = *reinterpret_cast<const float4 *>(c32 + 8 * (size_t)cn[c] + 4);
        const float xr = (ax - ox[c]) * prm.hx, yr = (ay - oy[c]) * prm.hy;
        ex = ((ex + r0.z) + (2.f * r1.x) * xr) + r1.y * yr;
        ey = ((ey + r0.w) + (2.f * r1.z) * yr) + r1.y * xr;
      }
      Ex = -ex / (float)cnt;
      Ey = -ey / (float)cnt;
    } else {
      const float xc = 1.f - ax, yc = 1.f - ay;
      const float w[4] = {xc * yc, ax * yc, ax * ay, xc * ay};
      Ex = 0.f;
      Ey = 0.f;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float2 ef = *reinterpret_cast<const float2 *>(c32 + 8 * (size_t)cn[c]);
        Ex = fmaf(w[c], ef.x, Ex);
        Ey = fmaf(w[c], ef.y, Ey);
      }
    }
    vx = fmaf(prm.qmdt, Ex, vx);
    vy = fmaf(prm.qmdt, Ey, vy);
    ax = fmaf(prm.dtx, vx, ax);
    if (AXI) {
      vt = fvz[p];
      double X = ((double)j + (double)ay) * prm.hyd + prm.dt * (double)vy, Y = prm.dt * (double)vt;
      if (X == 0.0) X = prm.hyd * (double)1.0e-5f;
      const double rn = sqrt(X * X + Y * Y), c = X / rn, sn = Y / rn;
      const double vr = c * (double)vy + sn * (double)vt, vtn = c * (double)vt - sn * (double)vy;
      vy = (float)vr;
      vt = (float)vtn;
      fvz[p] = vt;
      const double u = rn * prm.inv_hy, fu = floor(u);
      j = (int)fu;
      ay = (float)(u - fu);
      if (ay >= 1.f) { ay -= 1.f; ++j; }
    } else {
      ay = fmaf(prm.dty, vy, ay);
    }
    // re-home the offsets into [0, 1)
    const float dfx = floorf(ax), dfy = floorf(ay);
    ax -= dfx;
    ay -= dfy;
    i += (int)dfx;
    j += (int)dfy;
    if (ax >= 1.f) { ax -= 1.f; ++i; }
    if (ay >= 1.f) { ay -= 1.f; ++j; }
    // walls, in the order and with the comparisons of k_push: x <= xmin,
    // x > xmax, y < ymin, y > ymax on u = i + ax, v = j + ay
    auto rehome = [](float u, int *ii, float *aa) {
      const float f = floorf(u);
      *ii = (int)f;
      *aa = u - f;
      if (*aa >= 1.f) { *aa -= 1.f; ++*ii; }
    };
    if (i < 0 || (i == 0 && ax == 0.f)) {
      if (prm.wall[0] == PIC_WALL_REFLECT) { rehome(-((float)i + ax), &i, &ax); vx = -vx; }
      else lost = true;
    } else if (i > m.nex || (i == m.nex && ax > 0.f)) {
      if (prm.wall[1] == PIC_WALL_REFLECT) {
        int k2;
        float a2;
        rehome(-((float)(i - m.nex) + ax), &k2, &a2);
        i = m.nex + k2;
        ax = a2;
        vx = -vx;
      } else lost = true;
    } else if (j < 0) {
      if (prm.wall[2] == PIC_WALL_REFLECT) { rehome(-((float)j + ay), &j, &ay); vy = -vy; }
      else lost = true;
    } else if (j > m.ney || (j == m.ney && ay > 0.f)) {
      if (prm.wall[3] == PIC_WALL_REFLECT) {
        int k2;
        float a2;
        rehome(-((float)(j - m.ney) + ay), &k2, &a2);
        j = m.ney + k2;
        ay = a2;
        vy = -vy;
      } else lost = true;
    }
    // on the far walls: the last element, offset 1 (the clamp of GetParChg_2D.f90:143-149)
    if (i == m.nex && ax == 0.f) { i = m.nex - 1; ax = 1.f; }
    if (j == m.ney && ay == 0.f) { j = m.ney - 1; ay = 1.f; }
    if (!lost && (i < 0 || i >= m.nex || j < 0 || j >= m.ney)) {
      atomicAdd(s.bad, 1ull);  // still outside after one reflection
      lost = true;
    }
    if (!lost && m.elem_near[i * m.ney + j]) {
      const double X = m.xmin + ((double)i + (double)ax) * m.hx;
      const double Y = m.ymin + ((double)j + (double)ay) * m.hy;
      if (absorbed_by_object(X, Y)) lost = true;
    }
    fx[p] = ax;
    fy[p] = ay;
    fvx[p] = vx;
    fvy[p] = vy;
  }
  if (lost) {
    s.loc[p] = -1;
  } else {
    const int en = i * m.ney + j;
    if (prm.do_push) s.loc[p] = en;
    if (prm.do_deposit) {
      key = en;
      const double dx = ax, dy = ay, xc = 1.0 - dx, yc = 1.0 - dy;
      if (AXI) {
        const double jj = (double)j, den = 2.0 * jj + 1.0, beta = (j == 0) ? 0.75 : 1.0;
        const double lo = (yc * (den + dy)) / den, hi = (dy * (2.0 * jj + dy)) / den;
        W[0] = (xc * lo) * beta;
        W[1] = (dx * lo) * beta;
        W[2] = dx * hi;
        W[3] = xc * hi;
      } else {
        W[0] = xc * yc;
        W[1] = dx * yc;
        W[2] = dx * dy;
        W[3] = xc * dy;
      }
      const int n1 = i * m.nny + j;
      nodes[0] = n1;
      nodes[1] = n1 + m.nny;
      nodes[2] = n1 + m.nny + 1;
      nodes[3] = n1 + 1;
      if (prm.do_energy) {
        const double vz = (AXI && prm.do_push) ? (double)vt : (double)fvz[p], wx = vx, wy = vy;
        energy = ((((0.5 * prm.mass) * ((wx * wx + wy * wy) + vz * vz)) * prm.vref) * prm.vref) / PIC_JTOEV;
      }
    }
  }
}

template <bool AXI>
__global__ void __launch_bounds__(256, 4) k_push_mixed(MeshK m, const float *__restrict__ c32, PushM prm, SpK s) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
  const int lane = threadIdx.x & 31;
  int key = -1;
  double W[4] = {0, 0, 0, 0};
  int nodes[4] = {0, 0, 0, 0};
  double energy = 0.0;
  bool lost = false;
  if (p < s.n) {
    const int e = s.loc[p];
    if (e >= 0) {
      const float *fx = reinterpret_cast<const float *>(s.x), *fy = reinterpret_cast<const float *>(s.y);
      const float *fvx = reinterpret_cast<const float *>(s.vx), *fvy = reinterpret_cast<const float *>(s.vy);
      push_mixed_one<AXI>(m, c32, prm, s, p, e, fx[p], fy[p], fvx[p], fvy[p], key, W, nodes, energy, lost);
    }
  }
  warp_deposit<!AXI, !AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
  push_select(s, lane, key, p, pid);
}

// ---- the same push with the particle data staged through shared memory:
// persistent CTAs walk 256-particle tiles and copy the next S-1 tiles'
// element, offsets and velocities (5 KB a tile) with cp.async while they push
// the current one, so the DRAM reads of later tiles overlap the work on this
// one.  cp.async.wait_group is a hardware wait on the CTA's own copies.
constexpr int kPushTile = 256;
struct __align__(16) PushTile {
  int32_t loc[kPushTile];
  float ax[kPushTile], ay[kPushTile], vx[kPushTile], vy[kPushTile];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One thread's share of a tile's copy (blockDim.x == kPushTile): the tile
// is 5 arrays x 64 chunks of 16 B; thread t copies chunk t & 63 of array
// t >> 6, and threads below 64 also that chunk of the fifth array (vy).
struct TileCopy {
  const char *src0, *src1;
  int dst0, dst1, q;
};

__device__ __forceinline__ TileCopy tile_copy_of(const SpK &s) {
  TileCopy c;
  const int a = threadIdx.x >> 6;
  c.q = threadIdx.x & 63;
  c.src0 = reinterpret_cast<const char *>(a == 0 ? (const void *)s.loc
                                          : a == 1 ? (const void *)s.x
                                          : a == 2 ? (const void *)s.y
                                                   : (const void *)s.vx);
  c.src1 = reinterpret_cast<const char *>(s.vy);
  c.dst0 = a * 4 * kPushTile + 16 * c.q;
  c.dst1 = 4 * 4 * kPushTile + 16 * c.q;
  return c;
}

// the tile starting at particle `base`; chunks past the end read only their
// valid bytes (zero fill), none when empty
__device__ __forceinline__ void push_tile_load(PushTile *T, const TileCopy &c, int64_t n, int64_t base) {
  const int64_t first = base + 4 * c.q;
  const int valid = (int)max((int64_t)0, min((int64_t)4, n - first));
  const int64_t off = valid > 0 ? 4 * first : 0;
  char *t = reinterpret_cast<char *>(T);
  cp_async16(t + c.dst0, c.src0 + off, 4 * valid);
  if (threadIdx.x < 64) cp_async16(t + c.dst1, c.src1 + off, 4 * valid);
}

template <int S, int MINB = 4, bool AXI = false>
__global__ void __launch_bounds__(256, MINB) k_push_mixed_tiled(MeshK m, const float *__restrict__ c32, PushM prm,
                                                              SpK s, int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char push_smem[];
  PushTile *T = reinterpret_cast<PushTile *>(push_smem);
  const int lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
  const TileCopy cp = tile_copy_of(s);
#pragma unroll
  for (int k = 0; k < S - 1; ++k) {
    const int64_t t = blockIdx.x + k * G;
    if (t < ntiles) push_tile_load(&T[k], cp, s.n, t * kPushTile);
    cp_async_commit();
  }
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int64_t tn = t + (S - 1) * G;
    if (tn < ntiles) push_tile_load(&T[(it + S - 1) % S], cp, s.n, tn * kPushTile);
    cp_async_commit();
    cp_async_wait<S - 1>();  // this thread's copies of tile t are complete
    __syncthreads();         // and every thread's
    const PushTile &C = T[it % S];
    const int64_t p = t * kPushTile + threadIdx.x;
    const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
    int key = -1;
    double W[4] = {0, 0, 0, 0};
    int nodes[4] = {0, 0, 0, 0};
    double energy = 0.0;
    bool lost = false;
    if (p < s.n) {
      const int e = C.loc[threadIdx.x];
      if (e >= 0)
        push_mixed_one<AXI>(m, c32, prm, s, p, e, C.ax[threadIdx.x], C.ay[threadIdx.x], C.vx[threadIdx.x],
                            C.vy[threadIdx.x], key, W, nodes, energy, lost);
    }
    warp_deposit<!AXI, !AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
    push_select(s, lane, key, p, pid);
    __syncthreads();  // tile t is read before its stage is refilled
  }
  cp_async_wait<0>();
}

// ---- the FP64 push with the particle data staged through shared memory,
// as k_push_mixed_tiled: persistent CTAs walk 256-particle tiles and copy the
// next S-1 tiles' element and FP64 position and velocity (9 KB a tile) with
// cp.async while they push the current one.  The per-particle code is
// k_push's (push_fp64_one), so the results are the same bits.
struct __align__(16) PushTile64 {
  double x[kPushTile], y[kPushTile], vx[kPushTile], vy[kPushTile];
  int32_t loc[kPushTile];
};
// 16-byte chunks of a tile: 4 x 128 for the doubles, 64 for the elements
constexpr int kTile64Chunks = 4 * 128 + 64;

__device__ __forceinline__ void push_tile64_chunk(PushTile64 *T, const SpK &s, int64_t base, int c) {
  char *t = reinterpret_cast<char *>(T);
  if (c < 512) {  // array c >> 7, chunk c & 127 (two doubles)
    const int a = c >> 7, q = c & 127;
    const double *arr = a == 0 ? s.x : a == 1 ? s.y : a == 2 ? s.vx : s.vy;
    const int64_t first = base + 2 * q;
    const int valid = (int)max((int64_t)0, min((int64_t)2, s.n - first));
    cp_async16(t + 16 * c, reinterpret_cast<const char *>(arr) + (valid > 0 ? 8 * first : 0), 8 * valid);
  } else {  // element ids, chunk c - 512 (four int32)
    const int q = c - 512;
    const int64_t first = base + 4 * q;
    const int valid = (int)max((int64_t)0, min((int64_t)4, s.n - first));
    cp_async16(t + 4 * 8 * kPushTile + 16 * q, reinterpret_cast<const char *>(s.loc) + (valid > 0 ? 4 * first : 0),
               4 * valid);
  }
}

__device__ __forceinline__ void push_tile64_load(PushTile64 *T, const SpK &s, int64_t base) {
  for (int c = threadIdx.x; c < kTile64Chunks; c += kPushTile) push_tile64_chunk(T, s, base, c);
}

template <int S, bool AXI>
__global__ void __launch_bounds__(256, 4) k_push_tiled(MeshK m, FieldK f, PushK prm, SpK s, int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char push_smem[];
  PushTile64 *T = reinterpret_cast<PushTile64 *>(push_smem);
  const int lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
#pragma unroll
  for (int k = 0; k < S - 1; ++k) {
    const int64_t t = blockIdx.x + k * G;
    if (t < ntiles) push_tile64_load(&T[k], s, t * kPushTile);
    cp_async_commit();
  }
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int64_t tn = t + (S - 1) * G;
    if (tn < ntiles) push_tile64_load(&T[(it + S - 1) % S], s, tn * kPushTile);
    cp_async_commit();
    cp_async_wait<S - 1>();  // this thread's copies of tile t are complete
    __syncthreads();         // and every thread's
    const PushTile64 &C = T[it % S];
    const int64_t p = t * kPushTile + threadIdx.x;
    const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
    int key = -1;
    double W[4] = {0, 0, 0, 0};
    int nodes[4] = {0, 0, 0, 0};
    double energy = 0.0;
    bool lost = false;
    if (p < s.n) {
      const int e = C.loc[threadIdx.x];
      if (e >= 0)
        push_fp64_one<AXI>(m, f, prm, s, p, e, C.x[threadIdx.x], C.y[threadIdx.x], C.vx[threadIdx.x],
                           C.vy[threadIdx.x], key, W, nodes, energy, lost);
    }
    warp_deposit<!AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
    push_select(s, lane, key, p, pid);
    __syncthreads();  // tile t is read before its stage is refilled
  }
  cp_async_wait<0>();
}

// FP64 absolute particles (staging set) -> FP32 offsets inside the located
// element and FP32 velocities (live set).  Slots with loc < 0 are copied as 0.
// FP64 push with bulk-copied tiles: one thread issues five 1-D
// cp.async.bulk copies per 256-particle tile (x, y, vx, vy: 2 KB each; the
// elements: 1 KB), which complete on the stage's mbarrier; the other threads
// only wait on it, so no thread computes copy addresses.  Whole tiles are
// copied, the last one too: the particle arrays are allocated in whole
// tiles and slots at or beyond n are never used.  The wait is bounded: a
// tile not complete after `limit` polls sets *s.fail, and the CTA leaves at
// the next tile boundary.  The per-particle code is k_push's, bit for bit.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}

__device__ __forceinline__ void push_tile64_bulk(PushTile64 *T, uint64_t *b, const SpK &s, int64_t base) {
  mbar_expect_tx(b, (unsigned)sizeof(PushTile64));
  bulk_g2s(T->x, s.x + base, 8 * kPushTile, b);
  bulk_g2s(T->y, s.y + base, 8 * kPushTile, b);
  bulk_g2s(T->vx, s.vx + base, 8 * kPushTile, b);
  bulk_g2s(T->vy, s.vy + base, 8 * kPushTile, b);
  bulk_g2s(T->loc, s.loc + base, 4 * kPushTile, b);
}

template <int S, bool AXI, int MINB = 4>
__global__ void __launch_bounds__(256, MINB) k_push_bulk(MeshK m, FieldK f, PushK prm, SpK s, int64_t ntiles,
                                                      long long limit, int skip_copies) {
  extern __shared__ __align__(16) unsigned char push_smem[];
  PushTile64 *T = reinterpret_cast<PushTile64 *>(push_smem);
  uint64_t *bar = reinterpret_cast<uint64_t *>(push_smem + S * sizeof(PushTile64));
  __shared__ int s_fail;
  __shared__ SelBuf sel_buf;
  const int lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < S; ++k) mbar_init(&bar[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
    sel_buf.n = 0;
#pragma unroll
    for (int k = 0; k < S - 1; ++k) {
      const int64_t t = blockIdx.x + k * G;
      if (t < ntiles && !skip_copies) push_tile64_bulk(&T[k], &bar[k], s, t * kPushTile);
    }
  }
  __syncthreads();
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += G, ++it) {
    if (s_fail) break;  // read after the CTA barrier that ends each tile: the same for every thread
    if (threadIdx.x == 0) {
      const int64_t tn = t + (S - 1) * G;
      // the stage refilled here was read in the previous tile, before its
      // closing barrier; order those reads before the copy's writes
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      if (tn < ntiles && !skip_copies)
        push_tile64_bulk(&T[(it + S - 1) % S], &bar[(it + S - 1) % S], s, tn * kPushTile);
    }
    const int st = it % S;
    bool ready = false;
    for (long long k = 0; k < limit && !ready; ++k) ready = mbar_try_wait(&bar[st], (unsigned)((it / S) & 1));
    if (!ready) {
      s_fail = 1;
      atomicAdd(s.fail, 1ull);
    }
    const PushTile64 &C = T[st];
    const int64_t p = t * kPushTile + threadIdx.x;
    const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
    int key = -1;
    double W[4] = {0, 0, 0, 0};
    int nodes[4] = {0, 0, 0, 0};
    double energy = 0.0;
    bool lost = false;
    if (ready && p < s.n) {
      const int e = C.loc[threadIdx.x];
      if (e >= 0)
        push_fp64_one<AXI>(m, f, prm, s, p, e, C.x[threadIdx.x], C.y[threadIdx.x], C.vx[threadIdx.x],
                           C.vy[threadIdx.x], key, W, nodes, energy, lost);
    }
    warp_deposit<!AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
    push_select_cta(s, key, p, pid, sel_buf);
    __syncthreads();  // tile t is read before its stage is refilled
  }
  push_select_flush(s, sel_buf);
}

// The mixed-precision push with bulk-copied tiles (elements and FP32
// offsets and velocities: five 1 KB copies a tile), as k_push_bulk.
__device__ __forceinline__ void push_tile_bulk(PushTile *T, uint64_t *b, const SpK &s, int64_t base) {
  mbar_expect_tx(b, (unsigned)sizeof(PushTile));
  bulk_g2s(T->loc, s.loc + base, 4 * kPushTile, b);
  bulk_g2s(T->ax, reinterpret_cast<const float *>(s.x) + base, 4 * kPushTile, b);
  bulk_g2s(T->ay, reinterpret_cast<const float *>(s.y) + base, 4 * kPushTile, b);
  bulk_g2s(T->vx, reinterpret_cast<const float *>(s.vx) + base, 4 * kPushTile, b);
  bulk_g2s(T->vy, reinterpret_cast<const float *>(s.vy) + base, 4 * kPushTile, b);
}

template <int S, int MINB, bool AXI>
__global__ void __launch_bounds__(256, MINB) k_push_mixed_bulk(MeshK m, const float *__restrict__ c32, PushM prm,
                                                             SpK s, int64_t ntiles, long long limit,
                                                             int skip_copies) {
  extern __shared__ __align__(16) unsigned char push_smem[];
  PushTile *T = reinterpret_cast<PushTile *>(push_smem);
  uint64_t *bar = reinterpret_cast<uint64_t *>(push_smem + S * sizeof(PushTile));
  __shared__ int s_fail;
  __shared__ SelBuf sel_buf;
  const int lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < S; ++k) mbar_init(&bar[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
    sel_buf.n = 0;
#pragma unroll
    for (int k = 0; k < S - 1; ++k) {
      const int64_t t = blockIdx.x + k * G;
      if (t < ntiles && !skip_copies) push_tile_bulk(&T[k], &bar[k], s, t * kPushTile);
    }
  }
  __syncthreads();
  int it = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += G, ++it) {
    if (s_fail) break;  // read after the CTA barrier that ends each tile: the same for every thread
    if (threadIdx.x == 0) {
      const int64_t tn = t + (S - 1) * G;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      if (tn < ntiles && !skip_copies)
        push_tile_bulk(&T[(it + S - 1) % S], &bar[(it + S - 1) % S], s, tn * kPushTile);
    }
    const int st = it % S;
    bool ready = false;
    for (long long k = 0; k < limit && !ready; ++k) ready = mbar_try_wait(&bar[st], (unsigned)((it / S) & 1));
    if (!ready) {
      s_fail = 1;
      atomicAdd(s.fail, 1ull);
    }
    const PushTile &C = T[st];
    const int64_t p = t * kPushTile + threadIdx.x;
    const uint32_t pid = push_select_id(s, p);  // issued early: used after the push
    int key = -1;
    double W[4] = {0, 0, 0, 0};
    int nodes[4] = {0, 0, 0, 0};
    double energy = 0.0;
    bool lost = false;
    if (ready && p < s.n) {
      const int e = C.loc[threadIdx.x];
      if (e >= 0)
        push_mixed_one<AXI>(m, c32, prm, s, p, e, C.ax[threadIdx.x], C.ay[threadIdx.x], C.vx[threadIdx.x],
                            C.vy[threadIdx.x], key, W, nodes, energy, lost);
    }
    warp_deposit<!AXI, !AXI>(s, lane, key, W, nodes, energy, lost, prm.do_deposit, prm.do_energy);
    push_select_cta(s, key, p, pid, sel_buf);
    __syncthreads();  // tile t is read before its stage is refilled
  }
  push_select_flush(s, sel_buf);
}

__global__ void k_to_mixed(MeshK m, const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ vx, const double *__restrict__ vy,
                           const double *__restrict__ vz, const int32_t *__restrict__ loc, float *__restrict__ ox,
                           float *__restrict__ oy, float *__restrict__ ovx, float *__restrict__ ovy,
                           float *__restrict__ ovz, int64_t n) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int e = loc[p];
  float a = 0.f, b = 0.f;
  if (e >= 0) {
    const int i = elem_column(m, e), j = e - i * m.ney;
    a = (float)((x[p] - m.xs[i]) / (m.xs[i + 1] - m.xs[i]));
    b = (float)((y[p] - m.ys[j]) / (m.ys[j + 1] - m.ys[j]));
    a = fminf(fmaxf(a, 0.f), 1.f);
    b = fminf(fmaxf(b, 0.f), 1.f);
  }
  ox[p] = a;
  oy[p] = b;
  ovx[p] = (float)vx[p];
  ovy[p] = (float)vy[p];
  ovz[p] = (float)vz[p];
}

// FP32 live set -> FP64 absolute positions and velocities (staging set).
__global__ void k_from_mixed(MeshK m, const float *__restrict__ ax, const float *__restrict__ ay,
                             const float *__restrict__ avx, const float *__restrict__ avy,
                             const float *__restrict__ avz, const int32_t *__restrict__ loc, double *__restrict__ x,
                             double *__restrict__ y, double *__restrict__ vx, double *__restrict__ vy,
                             double *__restrict__ vz, int64_t n) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int e = loc[p];
  double X = 0.0, Y = 0.0;
  if (e >= 0) {
    const int i = elem_column(m, e), j = e - i * m.ney;
    X = m.xmin + ((double)i + (double)ax[p]) * m.hx;
    Y = m.ymin + ((double)j + (double)ay[p]) * m.hy;
  }
  x[p] = X;
  y[p] = Y;
  vx[p] = avx[p];
  vy[p] = avy[p];
  vz[p] = avz[p];
}

// ----------------------------------------------------------------------------
// field kernels
// ----------------------------------------------------------------------------

struct RhoK {
  const unsigned long long *q[PIC_MAX_SPECIES], *e[PIC_MAX_SPECIES];
  double *rho_s[PIC_MAX_SPECIES], *ek_s[PIC_MAX_SPECIES], *ek_tot[PIC_MAX_SPECIES];
  double wq[PIC_MAX_SPECIES], w[PIC_MAX_SPECIES];
  int ns;
  double L_ref, n_ref;
  int energy;  // update the per-node mean energy (diagnostic steps)
  int axi;     // delta = 1
};

// GetParChg_2D.f90:869-911: rho_s = Weight*qs*sum/L_ref/L_ref/n_ref/V; on
// energy steps the mean energy per particle (eV) Ek_s = sum(W*E)/sum(W) and
// the energy density Ek_tot = Weight*sum(W*E)/L_ref/L_ref/n_ref/V per node.
__global__ void k_rho(RhoK r, const double *__restrict__ vol, double *__restrict__ rho, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  double acc = 0.0;
  double V = vol[n];
  for (int s = 0; s < r.ns; ++s) {
    double cnt = (double)(long long)r.q[s][n] * (1.0 / PIC_Q_SCALE);
    double esum = (double)(long long)r.e[s][n] * (1.0 / PIC_E_SCALE);
    // one more 1/L_ref for delta = 1 (GetParChg_2D.f90:900-904): the dual
    // volume is then a volume, not an area
    double t = ((r.wq[s] * cnt) / r.L_ref) / r.L_ref;
    if (r.axi) t = t / r.L_ref;
    double rs = (t / r.n_ref) / V;
    r.rho_s[s][n] = rs;
    if (r.energy) {
      r.ek_s[s][n] = (cnt != 0.0) ? esum / cnt : 0.0;
      double te = ((r.w[s] * esum) / r.L_ref) / r.L_ref;
      if (r.axi) te = te / r.L_ref;
      r.ek_tot[s][n] = (te / r.n_ref) / V;
    }
    acc = acc + rs;
  }
  rho[n] = acc;
}

struct RhsK {
  const double *rho, *mass_q1, *ife_mass, *rhs_fix, *phi_dir, *xt_val;
  const double *mass_rows;  // delta = 1: [ney][16] r-weighted Q1 load matrix per element row, else null
  const int32_t *node_type, *element_index, *xt_ptr, *xt_col;
  double *b;
  int nnx, nny, ney;
  int64_t nn;
};

// b = M*rho - rhs_FIX - A_xt*phi_D on the full node grid (0 on Dirichlet nodes).
__global__ void k_rhs(RhsK k) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  int u = k.node_type[n];
  if (u <= 0) {
    k.b[n] = 0.0;
    return;
  }
  int i = (int)(n / k.nny), j = (int)(n - (int64_t)i * k.nny);
  // adjacent elements in element order and this node's corner in each
  const int di[4] = {-1, -1, 0, 0}, dj[4] = {-1, 0, -1, 0}, corner[4] = {2, 1, 3, 0};
  double acc = 0.0;
  for (int t = 0; t < 4; ++t) {
    int ei = i + di[t], ej = j + dj[t];
    if (ei < 0 || ej < 0 || ei >= k.nnx - 1 || ej >= k.nny - 1) continue;
    int e = ei * k.ney + ej;
    int id = k.element_index[e];
    const double *M = (id > 0)       ? (k.ife_mass + 16 * (size_t)(id - 1))
                      : k.mass_rows ? (k.mass_rows + 16 * (size_t)ej)
                                    : k.mass_q1;
    int n1 = ei * k.nny + ej;
    double R0 = k.rho[n1], R1 = k.rho[n1 + k.nny], R2 = k.rho[n1 + k.nny + 1], R3 = k.rho[n1 + 1];
    const double *Mr = M + 4 * corner[t];
    double el = ((Mr[0] * R0 + Mr[1] * R1) + Mr[2] * R2) + Mr[3] * R3;
    acc = acc + el;
  }
  double ebc = 0.0;
  for (int q = k.xt_ptr[u - 1]; q < k.xt_ptr[u]; ++q) ebc = ebc + k.phi_dir[k.xt_col[q]] * k.xt_val[q];
  k.b[n] = (acc - k.rhs_fix[u - 1]) - ebc;
}

__constant__ double c_stencil[16][9];
__constant__ float c_stencil32[16][9];  // FP32 copy for the inner iterations of the mixed-precision FCG

struct PcgK {
  const int32_t *row_kind, *ex_cnt, *ex_col;
  const double *ex_val, *diag;
  const float *ex_val32;  // FP32 copy of ex_val
  double *x, *r, *w, *q, *b;
  const double *p_old;
  double *p_new;
  double *part;
  PcgState *st;
  const double *phi;
  const int32_t *node_type;
  int nny, n_mat;
  int64_t nn;
  int nb;
};

// y = A*v on the full grid for a node given a functor that returns v at a node.
template <class F>
__device__ __forceinline__ double row_apply(const PcgK &k, int64_t n, F v) {
  int kind = k.row_kind[n];
  if (kind < 0) return 0.0;
  double acc = 0.0;
  if (kind < k.n_mat) {
    const int64_t base = n - k.nny - 1;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc = fma(c_stencil[kind][3 * a + c], v(base + (int64_t)a * k.nny + c), acc);
  } else {
    // explicit row, padded to 9 slots so all loads are in flight together;
    // only the first cnt slots enter the sum, in CSR order
    const int rix = kind - k.n_mat;
    const int cnt = k.ex_cnt[rix];
    int32_t col[9];
    double val[9], xv[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      col[q] = k.ex_col[9 * (size_t)rix + q];
      val[q] = k.ex_val[9 * (size_t)rix + q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) xv[q] = v((int64_t)col[q]);
#pragma unroll
    for (int q = 0; q < 9; ++q)
      if (q < cnt) acc = fma(val[q], xv[q], acc);
  }
  return acc;
}

// r = b - A x0, w = r/diag, partials of b.b and r.w  (MY_PCG.f90:56-71, 77-83)
__global__ void __launch_bounds__(PIC_RED_THREADS) k_pcg_init(PcgK k) {
  double vb = 0.0, vrw = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= k.nn) continue;
    double bb = k.b[n];
    double ax = row_apply(k, n, [&](int64_t m) { return k.x[m]; });
    double rr = (k.row_kind[n] < 0) ? 0.0 : bb - ax;
    double ww = rr / k.diag[n];
    k.r[n] = rr;
    k.w[n] = ww;
    vb = fma(bb, bb, vb);
    vrw = fma(rr, ww, vrw);
  }
  double v[2] = {vb, vrw}, out[2];
  block_sum_canon<2>(v, out);
  if (threadIdx.x == 0) {
    k.part[blockIdx.x] = out[0];
    k.part[k.nb + blockIdx.x] = out[1];
  }
  if (arrive_last(&k.st->ticket)) {
    double tot[2];
    final_sum_canon<2>(k.part, k.nb, tot);
    if (threadIdx.x == 0) {
      PcgState *s = k.st;
      s->normRHS = tot[0];
      s->rho = tot[1];
      s->rho0 = 0.0;
      s->iter = 0;
      s->ierr = 0;
      s->done = 0;
      s->beta = 0.0;
      s->normR = 0.0;
      s->ticket = 0;
      if (!(tot[0] > 0.0)) {  // zero right-hand side: x = x0 already solves b=0 only if r=0
        s->done = 1;
        s->normR = 0.0;
      }
    }
  }
}

// Warm start from phi at unknown nodes (IFE_Solve_2D.f90:80-85).
__global__ void k_pcg_x0(PcgK k) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  k.x[n] = (k.node_type[n] > 0) ? k.phi[n] : 0.0;
}

// p = w (+ beta p), q = A p, partial p.q  (MY_PCG.f90:86-111)
__global__ void __launch_bounds__(PIC_RED_THREADS) k_pcg_dir(PcgK k) {
  const PcgState *s = k.st;
  if (*(volatile const int *)&s->done) return;
  const bool first = (*(volatile const int *)&s->iter) == 0;
  const double beta = *(volatile const double *)&s->beta;
  auto pn = [&](int64_t m) { return first ? k.w[m] : fma(beta, k.p_old[m], k.w[m]); };
  double vpq = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= k.nn) continue;
    double pv = pn(n);
    double qv = row_apply(k, n, pn);
    k.p_new[n] = pv;
    k.q[n] = qv;
    vpq = fma(pv, qv, vpq);
  }
  double v[1] = {vpq}, out[1];
  block_sum_canon<1>(v, out);
  if (threadIdx.x == 0) k.part[blockIdx.x] = out[0];
  if (arrive_last(&k.st->ticket)) {
    double tot[1];
    final_sum_canon<1>(k.part, k.nb, tot);
    if (threadIdx.x == 0) {
      PcgState *st = k.st;
      st->ticket = 0;
      if (tot[0] == 0.0) {
        st->ierr = 3;
        st->done = 1;
      } else {
        st->alpha = st->rho / tot[0];
      }
    }
  }
}

// x += alpha p, r -= alpha q, w = r/diag, partials r.r and r.w; convergence test
// normR/normRHS <= tol^2 (MY_PCG.f90:113-125).
__global__ void __launch_bounds__(PIC_RED_THREADS) k_pcg_upd(PcgK k) {
  PcgState *s = k.st;
  if (*(volatile int *)&s->done) return;
  const double alpha = *(volatile double *)&s->alpha;
  double vrr = 0.0, vrw = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= k.nn) continue;
    double pv = k.p_new[n];
    double xv = fma(alpha, pv, k.x[n]);
    double rv = fma(-alpha, k.q[n], k.r[n]);
    double wv = rv / k.diag[n];
    k.x[n] = xv;
    k.r[n] = rv;
    k.w[n] = wv;
    vrr = fma(rv, rv, vrr);
    vrw = fma(rv, wv, vrw);
  }
  double v[2] = {vrr, vrw}, out[2];
  block_sum_canon<2>(v, out);
  if (threadIdx.x == 0) {
    k.part[blockIdx.x] = out[0];
    k.part[k.nb + blockIdx.x] = out[1];
  }
  if (arrive_last(&s->ticket)) {
    double tot[2];
    final_sum_canon<2>(k.part, k.nb, tot);
    if (threadIdx.x == 0) {
      s->ticket = 0;
      s->normR = tot[0];
      s->rho0 = s->rho;
      s->rho = tot[1];
      s->iter = s->iter + 1;
      if (s->normR / s->normRHS <= s->tol2) {
        s->done = 1;
      } else if (s->iter >= s->maxit) {
        s->ierr = 1;
        s->done = 1;
      } else if (s->rho0 == 0.0) {
        s->ierr = 2;
        s->done = 1;
      } else {
        s->beta = s->rho / s->rho0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Persistent Jacobi-PCG: one cooperative launch per solve.  Every CTA owns
// the 1024-node chunks blockIdx.x, blockIdx.x + gridDim.x, ...; per iteration
// two grid barriers separate (A) direction + SpMV + p.q partials and (B) the
// x/r/w update + r.r, r.w partials.  Each CTA then reduces all chunk partials
// itself in the canonical order, so every CTA holds identical scalars and
// takes identical decisions.  Phase A and phase B partials live in separate
// arrays: a CTA that races ahead never overwrites partials that a slower CTA
// is still reducing.  Cross-CTA data is read with ld.global.cg (L2), never
// from a possibly stale L1 line.
// ---------------------------------------------------------------------------
struct PcgP {
  PcgK k;
  double *p0, *p1;
  double *partA, *partB;  // [nb], [2*nb]
  unsigned int *bar;      // [0] arrive count, [1] generation
  int *bar_err;
  long long spin_limit;
  unsigned int bar_extra; // arrivals expected beyond the grid (0; >0 only to test the timeout)
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int atom_add_release_gpu(unsigned int *p, unsigned int v) {
  unsigned int o;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(o) : "l"(p), "r"(v) : "memory");
  return o;
}

// Grid-wide barrier on a monotonic arrival counter: thread 0 of every CTA
// adds 1 with release semantics (after the CTA barrier, so the whole CTA's
// writes are ordered before it) and polls with acquire loads until the count
// reaches the end of its round.  The wait is bounded: after `limit` polls the
// CTA records the timeout in *err and leaves; every CTA then exits the solve,
// so a lost CTA ends the kernel with an error status instead of a hang.
// Thread 0 reads the error word once and hands it to the CTA through shared
// memory (one global round trip per barrier instead of one per warp).
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, int *err, long long limit,
                                             unsigned int extra) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int n = gridDim.x + extra;
    unsigned int t = atom_add_release_gpu(bar, 1u);
    unsigned int target = (t / n + 1u) * n;
    long long spins = 0;
    while ((int)(ld_acquire_gpu(bar) - target) < 0) {
      if (++spins > limit) {
        atomicExch(err, 1);
        break;
      }
    }
    s_ok = *(volatile int *)err == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// The persistent solver runs CTAs of PIC_RED_CHUNK (1024) threads, one chunk
// node per thread, so all loads of a phase are in flight together.  Products
// are staged in shared memory and the first PIC_RED_THREADS threads then sum
// them exactly as the canonical reduction does (items t, t+256, t+512, t+768
// in order, xor butterfly, warp sums in order).
constexpr int kWide = PIC_RED_CHUNK;

// Canonical partial of a chunk: NV dot products sum_i fma(a_k[i], b_k[i], .)
// over the first nvalid entries; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void chunk_dots(const double (*a)[kWide], const double (*b)[kWide], int nvalid,
                                           double *out) {
  __shared__ double ws[NV][PIC_RED_THREADS / 32];
  if (threadIdx.x < PIC_RED_THREADS) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double acc = 0.0;
      for (int it = 0; it < PIC_RED_ITEMS; ++it) {
        int i = it * PIC_RED_THREADS + threadIdx.x;
        if (i < nvalid) acc = fma(a[k][i], b[k][i], acc);
      }
      for (int off = 16; off > 0; off >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
      if ((threadIdx.x & 31) == 0) ws[k][threadIdx.x >> 5] = acc;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int q = 0; q < PIC_RED_THREADS / 32; ++q) t = t + ws[k][q];
      out[k] = t;
    }
  __syncthreads();
}

// Sum of nb chunk partials in the canonical order, broadcast to every thread.
template <int NV>
__device__ __forceinline__ void final_sum_wide(const double *part, int nb, double *out_all) {
  __shared__ double ws[NV][PIC_RED_THREADS / 32];
  __shared__ double bc[NV];
  if (threadIdx.x < PIC_RED_THREADS) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double a = 0.0;
      for (int b = threadIdx.x; b < nb; b += PIC_RED_THREADS) a = a + __ldcg(part + (size_t)k * nb + b);
      for (int off = 16; off > 0; off >>= 1) a = a + __shfl_xor_sync(0xffffffffu, a, off);
      if ((threadIdx.x & 31) == 0) ws[k][threadIdx.x >> 5] = a;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int q = 0; q < PIC_RED_THREADS / 32; ++q) t = t + ws[k][q];
      bc[k] = t;
    }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) out_all[k] = bc[k];
  __syncthreads();
}

__global__ void __launch_bounds__(kWide, 1) k_pcg_persist(PcgP P) {
  const PcgK &k = P.k;
  PcgState *S = k.st;
  __shared__ double sa[2][kWide], sb[2][kWide];
  double rho = __ldcg(&S->rho), normRHS = __ldcg(&S->normRHS);
  const double tol2 = S->tol2;
  const int maxit = S->maxit;
  int done = __ldcg(&S->done), iter = 0, ierr = 0, parity = 0;
  double beta = 0.0, normR = 0.0, rho0 = 0.0;
  bool ok = true;
  while (!done) {
    const double *pold = parity ? P.p1 : P.p0;
    double *pnew = parity ? P.p0 : P.p1;
    const bool first = iter == 0;
    auto pn = [&](int64_t m) {
      double wm = __ldcg(k.w + m);
      return first ? wm : fma(beta, __ldcg(pold + m), wm);
    };
    // (A) p = w + beta p, q = A p, chunk partials of p.q
    for (int c = blockIdx.x; c < k.nb; c += gridDim.x) {
      const int64_t base = (int64_t)c * kWide;
      const int nvalid = (int)min((int64_t)kWide, k.nn - base);
      const int64_t n = base + threadIdx.x;
      double pv = 0.0, qv = 0.0;
      if (threadIdx.x < nvalid) {
        pv = pn(n);
        qv = row_apply(k, n, pn);
        pnew[n] = pv;
        k.q[n] = qv;
      }
      sa[0][threadIdx.x] = pv;
      sb[0][threadIdx.x] = qv;
      __syncthreads();
      double part[1];
      chunk_dots<1>(sa, sb, nvalid, part);
      if (threadIdx.x == 0) P.partA[c] = part[0];
    }
    if (!(ok = grid_barrier(P.bar, P.bar_err, P.spin_limit, P.bar_extra))) break;
    double pq;
    final_sum_wide<1>(P.partA, k.nb, &pq);
    if (pq == 0.0) {
      ierr = 3;
      break;
    }
    const double alpha = rho / pq;
    // (B) x += alpha p, r -= alpha q, w = r/diag, chunk partials of r.r and r.w
    for (int c = blockIdx.x; c < k.nb; c += gridDim.x) {
      const int64_t base = (int64_t)c * kWide;
      const int nvalid = (int)min((int64_t)kWide, k.nn - base);
      const int64_t n = base + threadIdx.x;
      double rv = 0.0, wv = 0.0;
      if (threadIdx.x < nvalid) {
        double xv = fma(alpha, pnew[n], k.x[n]);
        rv = fma(-alpha, k.q[n], k.r[n]);
        wv = rv / k.diag[n];
        k.x[n] = xv;
        k.r[n] = rv;
        k.w[n] = wv;
      }
      sa[0][threadIdx.x] = rv;
      sb[0][threadIdx.x] = rv;
      sa[1][threadIdx.x] = rv;
      sb[1][threadIdx.x] = wv;
      __syncthreads();
      double part[2];
      chunk_dots<2>(sa, sb, nvalid, part);
      if (threadIdx.x == 0) {
        P.partB[c] = part[0];
        P.partB[k.nb + c] = part[1];
      }
    }
    if (!(ok = grid_barrier(P.bar, P.bar_err, P.spin_limit, P.bar_extra))) break;
    double tot[2];
    final_sum_wide<2>(P.partB, k.nb, tot);
    normR = tot[0];
    rho0 = rho;
    rho = tot[1];
    ++iter;
    if (normR / normRHS <= tol2) done = 1;
    else if (iter >= maxit) { ierr = 1; done = 1; }
    else if (rho0 == 0.0) { ierr = 2; done = 1; }
    else beta = rho / rho0;
    parity ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->iter = iter;
    S->ierr = ok ? ierr : 4;
    S->normR = normR;
    S->rho = rho;
    S->done = 1;
  }
}

// ---------------------------------------------------------------------------
// Shared-memory-resident persistent Jacobi-PCG.  CTA b owns the contiguous
// chunks [c0, c1) (nodes [n0, n1), at most kSmemChunks chunks) and keeps
// x, r, q, diag, p_new of its nodes and a window [n0-H, n1+H) of w and p
// (H = nny+1, the reach of a 3x3 stencil) in shared memory for the whole
// solve.  Per iteration only the H-wide boundary strips of w and p cross
// L2: published before the second barrier, read after it.  Same chunk
// partials and canonical sums as the other PCG kernels, so the same bits.
// ---------------------------------------------------------------------------
constexpr int kSmemChunks = 2;

struct PcgS {
  PcgK k;
  double *w_g, *p_g;      // boundary-strip exchange (full-grid arrays)
  double *partA, *partB;
  unsigned int *bar;
  int *bar_err;
  long long spin_limit;
  unsigned int bar_extra;
  int H;                  // halo width in nodes
};

__host__ __device__ inline void smem_range(int b, int G, int nb, int *c0, int *c1) {
  *c0 = (int)((int64_t)b * nb / G);
  *c1 = (int)((int64_t)(b + 1) * nb / G);
}

__global__ void __launch_bounds__(kWide, 1) k_pcg_smem(PcgS P) {
  extern __shared__ double smem[];
  const PcgK &k = P.k;
  PcgState *S = k.st;
  int c0, c1;
  smem_range(blockIdx.x, gridDim.x, k.nb, &c0, &c1);
  const int64_t n0 = (int64_t)c0 * kWide;
  const int64_t n1 = min((int64_t)c1 * kWide, k.nn);
  const int L = (int)(n1 - n0);
  const int H = P.H;
  const int64_t wbase = n0 - H;     // node of window slot 0
  const int W = L + 2 * H;
  double *win_w = smem, *win_p = win_w + W;
  double *s_x = win_p + W, *s_r = s_x + kSmemChunks * kWide, *s_q = s_r + kSmemChunks * kWide;
  double *s_d = s_q + kSmemChunks * kWide, *s_pn = s_d + kSmemChunks * kWide;
  // load own x, r, diag and the window of w (p is not read before iteration 1)
  for (int i = threadIdx.x; i < L; i += kWide) {
    s_x[i] = __ldcg(k.x + n0 + i);
    s_r[i] = __ldcg(k.r + n0 + i);
    s_d[i] = k.diag[n0 + i];
  }
  for (int i = threadIdx.x; i < W; i += kWide) {
    int64_t m = wbase + i;
    win_w[i] = (m >= 0 && m < k.nn) ? __ldcg(k.w + m) : 0.0;
    win_p[i] = 0.0;
  }
  __syncthreads();
  double rho = __ldcg(&S->rho), normRHS = __ldcg(&S->normRHS);
  const double tol2 = S->tol2;
  const int maxit = S->maxit;
  int done = __ldcg(&S->done), iter = 0, ierr = 0;
  double beta = 0.0, normR = 0.0, rho0 = 0.0;
  bool ok = true;
  while (!done) {
    const bool first = iter == 0;
    auto pn = [&](int64_t m) {
      const int64_t i = m - wbase;
      return first ? win_w[i] : fma(beta, win_p[i], win_w[i]);
    };
    // (A) p = w + beta p, q = A p, chunk partials of p.q
    for (int c = c0; c < c1; ++c) {
      const int off = (c - c0) * kWide;
      const int nvalid = (int)min((int64_t)kWide, n1 - (int64_t)c * kWide);
      const int64_t n = (int64_t)c * kWide + threadIdx.x;
      double pv = 0.0, qv = 0.0;
      if (threadIdx.x < nvalid) {
        pv = pn(n);
        qv = row_apply(k, n, pn);
      }
      s_pn[off + threadIdx.x] = pv;
      s_q[off + threadIdx.x] = qv;
      __syncthreads();
      double part[1];
      const double(*a)[kWide] = reinterpret_cast<const double(*)[kWide]>(s_pn + off);
      const double(*b)[kWide] = reinterpret_cast<const double(*)[kWide]>(s_q + off);
      chunk_dots<1>(a, b, nvalid, part);
      if (threadIdx.x == 0) P.partA[c] = part[0];
    }
    if (!(ok = grid_barrier(P.bar, P.bar_err, P.spin_limit, P.bar_extra))) break;
    double pq;
    final_sum_wide<1>(P.partA, k.nb, &pq);
    if (pq == 0.0) {
      ierr = 3;
      break;
    }
    const double alpha = rho / pq;
    // (B) x += alpha p, r -= alpha q, w = r/diag; window gets w and p for the
    // next iteration; boundary strips are published to L2
    for (int c = c0; c < c1; ++c) {
      const int off = (c - c0) * kWide;
      const int nvalid = (int)min((int64_t)kWide, n1 - (int64_t)c * kWide);
      const int i = off + threadIdx.x;
      if (threadIdx.x < nvalid) {
        const double pv = s_pn[i];
        s_x[i] = fma(alpha, pv, s_x[i]);
        const double rv = fma(-alpha, s_q[i], s_r[i]);
        const double wv = rv / s_d[i];
        s_r[i] = rv;
        s_q[i] = wv;  // q is dead after the update: reuse its slot for w
        win_w[H + i] = wv;
        win_p[H + i] = pv;
        if (i < H || i >= L - H) {
          P.w_g[n0 + i] = wv;
          P.p_g[n0 + i] = pv;
        }
      }
      __syncthreads();
      double part[2];
      const double *ra = s_r + off;
      const double *wa = s_q + off;
      // r.r and r.w in one canonical pass
      {
        __shared__ double ws2[2][PIC_RED_THREADS / 32];
        if (threadIdx.x < PIC_RED_THREADS) {
          double arr = 0.0, arw = 0.0;
          for (int it = 0; it < PIC_RED_ITEMS; ++it) {
            int j = it * PIC_RED_THREADS + threadIdx.x;
            if (j < nvalid) {
              arr = fma(ra[j], ra[j], arr);
              arw = fma(ra[j], wa[j], arw);
            }
          }
          for (int o2 = 16; o2 > 0; o2 >>= 1) {
            arr = arr + __shfl_xor_sync(0xffffffffu, arr, o2);
            arw = arw + __shfl_xor_sync(0xffffffffu, arw, o2);
          }
          if ((threadIdx.x & 31) == 0) {
            ws2[0][threadIdx.x >> 5] = arr;
            ws2[1][threadIdx.x >> 5] = arw;
          }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          double t0 = 0.0, t1 = 0.0;
          for (int q = 0; q < PIC_RED_THREADS / 32; ++q) {
            t0 = t0 + ws2[0][q];
            t1 = t1 + ws2[1][q];
          }
          part[0] = t0;
          part[1] = t1;
          P.partB[c] = part[0];
          P.partB[k.nb + c] = part[1];
        }
        __syncthreads();
      }
    }
    if (!(ok = grid_barrier(P.bar, P.bar_err, P.spin_limit, P.bar_extra))) break;
    // halo of the window from the neighbours' published strips
    for (int i = threadIdx.x; i < 2 * H; i += kWide) {
      const int slot = (i < H) ? i : (L + i);
      const int64_t m = wbase + slot;
      if (m >= 0 && m < k.nn) {
        win_w[slot] = __ldcg(P.w_g + m);
        win_p[slot] = __ldcg(P.p_g + m);
      }
    }
    double tot[2];
    final_sum_wide<2>(P.partB, k.nb, tot);
    normR = tot[0];
    rho0 = rho;
    rho = tot[1];
    ++iter;
    if (normR / normRHS <= tol2) done = 1;
    else if (iter >= maxit) { ierr = 1; done = 1; }
    else if (rho0 == 0.0) { ierr = 2; done = 1; }
    else beta = rho / rho0;
  }
  for (int i = threadIdx.x; i < L; i += kWide) k.x[n0 + i] = s_x[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->iter = iter;
    S->ierr = ok ? ierr : 4;
    S->normR = normR;
    S->rho = rho;
    S->done = 1;
  }
}

// U_fe_full from U_fe (IFE_Solve_2D.f90:240-247)
__global__ void k_phi_out(const double *__restrict__ x, const int32_t *__restrict__ node_type,
                          const double *__restrict__ phi_dir, double *__restrict__ phi, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  phi[n] = (node_type[n] > 0) ? x[n] : phi_dir[n];
}

// ---- operator and dot products used by flexible CG -------------------------

__global__ void k_spmv(PcgK k, const double *__restrict__ v, double *__restrict__ out) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  out[n] = row_apply(k, n, [&](int64_t m) { return v[m]; });
}

struct DotK {
  const double *a, *b, *c, *d;
  double *part, *out;
  unsigned int *ticket;
  int64_t nn;
  int nb;
};

// Canonical a.b and c.d (c may be NULL); the last block writes out[0..1].
__global__ void __launch_bounds__(PIC_RED_THREADS) k_dot(DotK k) {
  double v0 = 0.0, v1 = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= k.nn) continue;
    v0 = fma(k.a[n], k.b[n], v0);
    if (k.c) v1 = fma(k.c[n], k.d[n], v1);
  }
  double v[2] = {v0, v1}, out[2];
  block_sum_canon<2>(v, out);
  if (threadIdx.x == 0) {
    k.part[blockIdx.x] = out[0];
    k.part[k.nb + blockIdx.x] = out[1];
  }
  if (arrive_last(k.ticket)) {
    double tot[2];
    final_sum_canon<2>(k.part, k.nb, tot);
    if (threadIdx.x == 0) {
      k.out[0] = tot[0];
      k.out[1] = tot[1];
      *k.ticket = 0;
    }
  }
}

// r = b - q on unknown nodes, 0 on Dirichlet nodes
// The persistent FCG's set-up and judge in one launch each: r = b - A x (0
// on Dirichlet rows) over k_dot's item layout, with r.r (and b.b) summed in
// k_dot's order, so the numbers are those of k_pcg_x0 + k_spmv + k_fcg_r0 +
// k_dot.  init: x is the Dirichlet-filled phi, formed at every neighbour as
// k_pcg_x0 writes it, and the last block stores rhs = b.b, rr = best = r.r
// in the FCG state; otherwise x is read and rr = r.r is stored.
__global__ void __launch_bounds__(PIC_RED_THREADS) k_fcg_resid(PcgK k, unsigned int *__restrict__ ticket,
                                                               FcgState *__restrict__ S, int init) {
  double v0 = 0.0, v1 = 0.0;
  auto x0 = [&](int64_t m) { return k.node_type[m] > 0 ? k.phi[m] : 0.0; };
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    const int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= k.nn) continue;
    double q;
    if (init) {
      k.x[n] = x0(n);
      q = row_apply(k, n, x0);
    } else {
      q = row_apply(k, n, [&](int64_t m) { return k.x[m]; });
    }
    const double r = k.row_kind[n] < 0 ? 0.0 : k.b[n] - q;
    k.r[n] = r;
    v0 = fma(k.b[n], k.b[n], v0);
    v1 = fma(r, r, v1);
  }
  double v[2] = {v0, v1}, out[2];
  block_sum_canon<2>(v, out);
  if (threadIdx.x == 0) {
    k.part[blockIdx.x] = out[0];
    k.part[k.nb + blockIdx.x] = out[1];
  }
  if (arrive_last(ticket)) {
    double tot[2];
    final_sum_canon<2>(k.part, k.nb, tot);
    if (threadIdx.x == 0) {
      if (init) {
        S->rhs = tot[0];
        S->best = tot[1];
      }
      S->rr = tot[1];
      *ticket = 0;
    }
  }
}

__global__ void k_fcg_r0(const int32_t *__restrict__ row_kind, const double *__restrict__ b,
                         const double *__restrict__ q, double *__restrict__ r, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nn) r[n] = (row_kind[n] < 0) ? 0.0 : b[n] - q[n];
}

// ---- flexible CG, truncated FCG(m) (Notay, SIAM J. Sci. Comput. 22, 2000) --
// One iteration = preconditioner stage A (pre-smoothing, coarse correction),
// the learned stage (host callback, enqueued on the same stream), then
// k_fcg_post (post-smoothing + the A-orthogonalisation dots), k_fcg_dir (new
// direction + SpMV + p.q, p.r) and k_fcg_upd.  The new direction is
// A-orthogonalised against the last m <= PIC_FCG_MAX_WINDOW directions, kept
// in a ring of m + 1 slots P[j], Q[j] = A P[j] (one more than m, so the slot
// being written is never read as an old direction); m = 1 is FCG(1).  The
// scalars live in FcgState on the device; the host reads it once per chunk
// of iterations.  Reductions use the canonical block/final sums of the PCG.

struct FcgK {
  PcgK op;        // operator; op.w = z (final preconditioned residual), op.x, op.r
  double *P, *Q;  // ring [window + 1][nn]
  double *part;   // [PIC_FCG_MAX_WINDOW][nb]
  FcgState *s;    // NULL: no FCG bookkeeping (a bare preconditioner application)
  int slot, ring, window;  // ring slot of the new direction, ring size m + 1, window m
};

// The FCG scalars a kernel needs, read once per block (thread 0) and shared:
// every thread polling the same device word would queue on one L2 line.
struct FcgScal {
  int done, count;
  double alpha;
  double beta[PIC_FCG_MAX_WINDOW];
};

__device__ __forceinline__ void fcg_scalars(const FcgState *s, FcgScal *out, bool betas) {
  if (threadIdx.x == 0) {
    if (s) {
      out->done = *(volatile const int *)&s->done;
      out->count = *(volatile const int *)&s->count;
      out->alpha = *(volatile const double *)&s->alpha;
      if (betas)
        for (int t = 0; t < PIC_FCG_MAX_WINDOW; ++t) out->beta[t] = *(volatile const double *)&s->beta[t];
    } else {
      out->done = 0;
      out->count = 0;
      out->alpha = 0.0;
    }
  }
  __syncthreads();
}

// ring slot of the t-th previous direction (t = 1..count)
__device__ __forceinline__ int fcg_slot(const FcgK &k, int t) { return (k.slot - t + k.ring) % k.ring; }

// Pre-smoothing: zA = w D^-1 r and t = r - A zA, the product formed from
// r at the neighbours (no intermediate vector).  dinv = 1/diag (1 on
// Dirichlet nodes, where r is 0).
__global__ void k_pc_pre(PcgK k, const double *__restrict__ r, const double *__restrict__ dinv, double omega,
                         double *__restrict__ zA, double *__restrict__ t) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  if (k.row_kind[n] < 0) {
    zA[n] = 0.0;
    t[n] = 0.0;
    return;
  }
  auto z1 = [&](int64_t m) { return (omega * r[m]) * dinv[m]; };
  zA[n] = z1(n);
  t[n] = r[n] - row_apply(k, n, z1);
}

// t = r - A zA (the learned stage's input)
__global__ void k_pc_mid(PcgK k, const double *__restrict__ r, const double *__restrict__ zA,
                         double *__restrict__ t) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  t[n] = (k.row_kind[n] < 0) ? 0.0 : r[n] - row_apply(k, n, [&](int64_t m) { return zA[m]; });
}

// Post-smoothing of z3 = zA (+ y): zF = z3 + w D^-1 (r - A z3) (zF = z3 when
// smooth == 0), then, inside FCG, beta_t = -(zF.Q_t)/(P_t.Q_t) for the last
// `count` directions.
__global__ void __launch_bounds__(PIC_RED_THREADS) k_fcg_post(FcgK k, const double *__restrict__ r,
                                                              const double *__restrict__ zA,
                                                              const double *__restrict__ y,
                                                              const double *__restrict__ dinv, double omega,
                                                              int smooth, double *__restrict__ zF) {
  FcgState *s = k.s;
  __shared__ FcgScal sc;
  fcg_scalars(s, &sc, false);
  if (sc.done) return;
  const int cnt = sc.count;
  const int64_t nn = k.op.nn;
  auto z3 = [&](int64_t m) { return y ? zA[m] + y[m] : zA[m]; };
  double v[PIC_FCG_MAX_WINDOW];
#pragma unroll
  for (int q = 0; q < PIC_FCG_MAX_WINDOW; ++q) v[q] = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= nn) continue;
    double zf = 0.0;
    if (k.op.row_kind[n] >= 0) {
      zf = z3(n);
      if (smooth) zf = fma(omega * dinv[n], r[n] - row_apply(k.op, n, z3), zf);
    }
    zF[n] = zf;
#pragma unroll
    for (int q = 0; q < PIC_FCG_MAX_WINDOW; ++q)
      if (q < cnt) v[q] = fma(zf, k.Q[(size_t)fcg_slot(k, q + 1) * nn + n], v[q]);
  }
  if (!s || cnt == 0) return;
  double out[PIC_FCG_MAX_WINDOW];
  block_sum_canon<PIC_FCG_MAX_WINDOW>(v, out);
  if (threadIdx.x == 0)
    for (int q = 0; q < PIC_FCG_MAX_WINDOW; ++q) k.part[(size_t)q * k.op.nb + blockIdx.x] = out[q];
  if (arrive_last(&s->ticket)) {
    double tot[PIC_FCG_MAX_WINDOW];
    final_sum_canon<PIC_FCG_MAX_WINDOW>(k.part, k.op.nb, tot);
    if (threadIdx.x == 0) {
      s->ticket = 0;
      for (int q = 0; q < cnt; ++q) s->beta[q] = -tot[q] / s->pq_hist[fcg_slot(k, q + 1)];
    }
  }
}

// New direction P_new = z + sum_t beta_t P_t (on unknown nodes), formed at
// every neighbour on the fly for Q_new = A P_new; p.q and p.r; alpha = p.r/p.q.
__global__ void __launch_bounds__(PIC_RED_THREADS) k_fcg_dir(FcgK k) {
  FcgState *s = k.s;
  __shared__ FcgScal sc;
  fcg_scalars(s, &sc, true);
  if (sc.done) return;
  const int cnt = sc.count;
  const int64_t nn = k.op.nn;
  int off[PIC_FCG_MAX_WINDOW];
#pragma unroll
  for (int q = 0; q < PIC_FCG_MAX_WINDOW; ++q) off[q] = fcg_slot(k, q + 1);
  auto pn = [&](int64_t m) {
    if (k.op.row_kind[m] < 0) return 0.0;
    double v = k.op.w[m];
    for (int q = 0; q < cnt; ++q) v = fma(sc.beta[q], k.P[(size_t)off[q] * nn + m], v);
    return v;
  };
  double *Pn = k.P + (size_t)k.slot * nn, *Qn = k.Q + (size_t)k.slot * nn;
  double vpq = 0.0, vpr = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= nn) continue;
    const double pv = pn(n);
    const double qv = row_apply(k.op, n, pn);
    Pn[n] = pv;
    Qn[n] = qv;
    vpq = fma(pv, qv, vpq);
    vpr = fma(pv, k.op.r[n], vpr);
  }
  double v[2] = {vpq, vpr}, out[2];
  block_sum_canon<2>(v, out);
  if (threadIdx.x == 0) {
    k.part[blockIdx.x] = out[0];
    k.part[k.op.nb + blockIdx.x] = out[1];
  }
  if (arrive_last(&s->ticket)) {
    double tot[2];
    final_sum_canon<2>(k.part, k.op.nb, tot);
    if (threadIdx.x == 0) {
      s->ticket = 0;
      s->pq = tot[0];
      s->pr = tot[1];
      s->pq_hist[k.slot] = tot[0];
      s->count = min(s->count + 1, k.window);
      if (!(tot[0] > 0.0) || !(tot[1] == tot[1])) {
        s->ierr = 2;  // breakdown: M not positive on this residual
        s->done = 1;
      } else {
        s->alpha = tot[1] / tot[0];
      }
    }
  }
}

// x += alpha P_new, r -= alpha Q_new, r.r; convergence / cap / stall decisions.
__global__ void __launch_bounds__(PIC_RED_THREADS) k_fcg_upd(FcgK k) {
  FcgState *s = k.s;
  __shared__ FcgScal sc;
  fcg_scalars(s, &sc, false);
  if (sc.done) return;
  const double alpha = sc.alpha;
  const int64_t nn = k.op.nn;
  const double *pn = k.P + (size_t)k.slot * nn, *qn = k.Q + (size_t)k.slot * nn;
  double vrr = 0.0;
  for (int it = 0; it < PIC_RED_ITEMS; ++it) {
    int64_t n = (int64_t)blockIdx.x * PIC_RED_CHUNK + it * PIC_RED_THREADS + threadIdx.x;
    if (n >= nn) continue;
    k.op.x[n] = fma(alpha, pn[n], k.op.x[n]);
    double rv = fma(-alpha, qn[n], k.op.r[n]);
    k.op.r[n] = rv;
    vrr = fma(rv, rv, vrr);
  }
  double v[1] = {vrr}, out[1];
  block_sum_canon<1>(v, out);
  if (threadIdx.x == 0) k.part[blockIdx.x] = out[0];
  if (arrive_last(&s->ticket)) {
    double tot[1];
    final_sum_canon<1>(k.part, k.op.nb, tot);
    if (threadIdx.x == 0) {
      const double rr = tot[0];
      s->ticket = 0;
      s->rr = rr;
      s->iter = s->iter + 1;
      if (!(rr == rr)) {
        s->ierr = 4;
        s->done = 1;
      } else if (rr / s->rhs <= s->tol2) {
        s->done = 1;
      } else if (s->iter >= s->maxit) {
        s->ierr = 1;
        s->done = 1;
      } else {
        if (rr < s->best) {
          s->best = rr;
          s->best_iter = s->iter;
        }
        if (s->iter - s->best_iter > s->stall_window || rr > 1e6 * s->best) {
          s->ierr = 3;  // stalled
          s->done = 1;
        }
      }
    }
  }
}

// ---- persistent flexible CG (window 1, classical stages) -------------------
// The whole solve in one cooperative kernel of kWide-thread CTAs: per
// iteration six phases, separated by the bounded grid barrier of the
// persistent Jacobi-PCG.  Scalars (beta, alpha, r.r) are formed by every CTA
// from the chunk partials in the canonical order, so all CTAs take the same
// decisions.  Phases:
//   (A) x += alpha P, r' = r - alpha Q (previous direction; r ping-pongs,
//       r' is formed at the neighbours), r'.r', then pre-smoothing
//       zA = w D^-1 r', t = r' - A zA
//   (B) rc = P^T t                             (restriction, warp per coarse node)
//   (C) ec = Ac^-1 rc                          (GEMV, warp per row)
//   (D) zA += P ec                             (prolongation)
//   (E) zF = zA + w D^-1 (r - A zA), zF.Q_old  (post-smoothing)
//   (F) P_new = zF + beta P_old formed at the neighbours, Q_new = A P_new,
//       p.q, p.r
// Dot products are summed per thread over the CTA's chunks and once per CTA
// (cta_sum), so warps run through their chunks without CTA-wide waits; the
// order is fixed for a given grid, so the solve is deterministic.
// The convergence test on r'.r' follows phase A.  Without a coarse space
// phases B-D are skipped.  Loads after a grid barrier are plain (L1-cached)
// loads: the barrier's release/acquire pair orders every CTA's writes before
// them, and a stencil reads each value up to nine times, from L1.
// Sum over the CTA's kWide threads of NV values, in a fixed order (warp
// butterflies, then the warp sums in warp order); result valid in thread 0.
template <int NV>
__device__ __forceinline__ void cta_sum(double v[NV], double *out) {
  __shared__ double ws[NV][kWide / 32];
#pragma unroll
  for (int q = 0; q < NV; ++q)
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) ws[q][threadIdx.x >> 5] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = 0.0;
      for (int w = 0; w < kWide / 32; ++w) t += ws[q][w];
      out[q] = t;
    }
  __syncthreads();
}

template <class V>
struct FcgP {
  PcgK k;                        // operator (row kinds, FP64 and FP32 coefficients)
  V *x, *r, *r2;                 // solution, residual, second residual buffer (ping-pong)
  const V *dinv;
  V *zA, *t, *zF, *P0, *P1, *Q0, *Q1;
  double *part;                  // [4][grid] partials: F p.q, F p.r, A r.r, E zF.Q
  const __half *ainv;            // coarse inverse / ainv_scale, rows padded to ainv_ld (a multiple of 8)
  double ainv_scale;
  int ainv_ld;
  double *rc, *ec;
  int nnx, cs, ncx, ncy, coarse;
  MgK mg;                        // multigrid V-cycle (mg.L > 1) in place of the two-level space
  double omega;
  FcgState *s;
  unsigned int *bar;
  int *bar_err;
  long long spin_limit;
  unsigned int bar_extra;
};

__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }

// A*v for one node in the vector type: FP64 with the FP64 coefficients, FP32
// with their FP32 copies (same rows, same order).
template <class V, class F>
__device__ __forceinline__ V row_apply_v(const PcgK &k, int64_t n, F v) {
  if constexpr (sizeof(V) == sizeof(double)) {
    return row_apply(k, n, v);
  } else {
    const int kind = k.row_kind[n];
    if (kind < 0) return 0.0f;
    float acc = 0.0f;
    if (kind < k.n_mat) {
      const int64_t base = n - k.nny - 1;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc = fmaf(c_stencil32[kind][3 * a + c], v(base + (int64_t)a * k.nny + c), acc);
    } else {
      const int rix = kind - k.n_mat;
      const int cnt = k.ex_cnt[rix];
      int32_t col[9];
      float val[9], xv[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        col[q] = k.ex_col[9 * (size_t)rix + q];
        val[q] = k.ex_val32[9 * (size_t)rix + q];
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) xv[q] = v((int64_t)col[q]);
#pragma unroll
      for (int q = 0; q < 9; ++q)
        if (q < cnt) acc = fmaf(val[q], xv[q], acc);
    }
    return acc;
  }
}

// V = double: the FP64 solve.  V = float: the inner solve A e = r of the FP64
// iterative refinement (vectors and coefficients FP32, dot products and the
// coarse solve accumulated in FP64), started from e = 0.
// ec = Ainv rc with the scaled FP16 inverse: the CTA stages rc in shared
// memory (ainv_ld doubles, zero past nc) as eight planes, element 8q + k at
// k*nq + q, so that the lanes of a warp, each reading the eight coefficients
// of its 16-byte group q, read consecutive doubles of a plane (no bank
// conflicts); each warp takes rows, accumulating in FP64.  The caller
// separates it from the writes of rc by a grid barrier.
template <class V>
__device__ __forceinline__ void coarse_gemv(const FcgP<V> &F, int nc, double *s_rc, int gwarp, int nwarps,
                                            int lane) {
  const int ld = F.ainv_ld;
  const int nq = ld / 8;  // 16-byte groups of a row
  for (int i = threadIdx.x; i < ld; i += blockDim.x) s_rc[(i & 7) * nq + (i >> 3)] = i < nc ? __ldcg(F.rc + i) : 0.0;
  __syncthreads();
  for (int row = gwarp; row < nc; row += nwarps) {
    const uint4 *arow = reinterpret_cast<const uint4 *>(F.ainv + (size_t)row * ld);
    double acc = 0.0;
    // four loads in flight per lane before their FMAs (the row comes from
    // DRAM: one load at a time would make the row a chain of latencies)
    for (int q0 = lane; q0 < nq; q0 += 4 * 32) {
      uint4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + 32 * u;
        v[u] = q < nq ? __ldg(arow + q) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + 32 * u;
        if (q >= nq) break;
        const __half2 *h = reinterpret_cast<const __half2 *>(&v[u]);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float2 f = __half22float2(h[c]);
          acc = fma((double)f.x, s_rc[(2 * c) * nq + q], acc);
          acc = fma((double)f.y, s_rc[(2 * c + 1) * nq + q], acc);
        }
      }
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) F.ec[row] = acc * F.ainv_scale;
  }
}

template <class V>
__global__ void __launch_bounds__(kWide, 1) k_fcg_persist(FcgP<V> F) {
  extern __shared__ double fcg_smem[];  // the coarse right-hand side (coarse_gemv)
  const PcgK &k = F.k;
  FcgState *S = F.s;
  const int64_t nn = k.nn;
  const int nb = k.nb;
  const int G = gridDim.x;  // one partial per CTA and value, summed in CTA order
  const double rhs = S->rhs, tol2 = S->tol2, omega = F.omega;
  const V om = (V)omega;
  const int maxit = S->maxit, stall_window = S->stall_window;
  int iter = S->iter, ierr = 0, best_iter = S->best_iter;
  double rr = S->rr, best = S->best, pq_old = 0.0, alpha = 0.0;
  bool have_old = false, ok = true;
  int parity = 0;
  V *rc_ = F.r, *rn_ = F.r2;  // current residual, next residual
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gwarp = blockIdx.x * (kWide / 32) + warp, nwarps = gridDim.x * (kWide / 32);
  const int nc = F.ncx * F.ncy;
  auto barrier = [&]() { return grid_barrier(F.bar, F.bar_err, F.spin_limit, F.bar_extra); };
  // already converged (the state came from k_fcg_resid): nothing to do
  // (every CTA reads the same state)
  if (!(rhs > 0.0) || rr / rhs <= tol2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->ierr = 0;
      S->done = 1;
    }
    return;
  }
  for (;;) {
    // the previous direction (written last iteration), the new one
    const V *Pl = parity ? F.P0 : F.P1, *Ql = parity ? F.Q0 : F.Q1;
    V *Pn = parity ? F.P1 : F.P0, *Qn = parity ? F.Q1 : F.Q0;
    // (A) update with the previous direction, then pre-smoothing
    {
      const V *r = rc_, *Qp = Ql;
      const V a = (V)alpha;
      const bool upd = have_old;
      auto rnew = [&](int64_t m) { return upd ? vfma(-a, Qp[m], r[m]) : r[m]; };
      double acc_rr = 0.0;
      for (int c = blockIdx.x; c < nb; c += gridDim.x) {
        const int64_t base = (int64_t)c * kWide;
        const int nvalid = (int)min((int64_t)kWide, nn - base);
        const int64_t n = base + threadIdx.x;
        if (threadIdx.x < nvalid) {
          const V rv = rnew(n);
          if (upd) {
            F.x[n] = vfma(a, Pl[n], F.x[n]);
            rn_[n] = rv;
            acc_rr = fma((double)rv, (double)rv, acc_rr);
          }
          if (k.row_kind[n] < 0) {
            F.zA[n] = (V)0;
            F.t[n] = (V)0;
          } else {
            auto z1 = [&](int64_t m) { return (om * rnew(m)) * F.dinv[m]; };
            F.zA[n] = z1(n);
            F.t[n] = rv - row_apply_v<V>(k, n, z1);
          }
        }
      }
      if (upd) {
        double v[1] = {acc_rr}, o[1];
        cta_sum<1>(v, o);
        if (threadIdx.x == 0) F.part[2 * G + blockIdx.x] = o[0];
      }
      if (!(ok = barrier())) break;
      if (upd) {
        final_sum_wide<1>(F.part + 2 * G, G, &rr);
        ++iter;
        V *tmp = rc_;
        rc_ = rn_;
        rn_ = tmp;
        if (!(rr == rr)) { ierr = 4; break; }
        if (rr / rhs <= tol2) break;
        if (iter >= maxit) { ierr = 1; break; }
        if (rr < best) { best = rr; best_iter = iter; }
        if (iter - best_iter > stall_window || rr > 1e6 * best) { ierr = 3; break; }
      }
    }
    const V *r = rc_;
    const MgK &M = F.mg;
    if (M.L > 1) {
      // (B') multigrid V-cycle of t: restriction and down-sweeps, the dense
      // coarsest solve, up-sweeps; a grid barrier between dependent steps
      const int64_t gtid = (int64_t)blockIdx.x * kWide + threadIdx.x, gth = (int64_t)gridDim.x * kWide;
      for (int l = 1; l < M.L && ok; ++l) {
        const MgLevel &L = M.lv[l];
        const int64_t nl = (int64_t)L.nx * L.ny;
        const bool smoothed = l < M.L - 1;
        for (int64_t n = gtid; n < nl; n += gth) {
          if (l == 1) mg_restrict_node(L, F.t, F.nnx, k.nny, omega, smoothed, n);
          else mg_restrict_node(L, M.lv[l - 1].t, M.lv[l - 1].nx, M.lv[l - 1].ny, omega, smoothed, n);
        }
        if (!(ok = barrier())) break;
        if (smoothed) {
          // two nodes a thread at a time: both nodes' loads ahead of the stores
          for (int64_t n = gtid; n < nl; n += 2 * gth) {
            const int64_t n2 = n + gth;
            const double a = mg_smooth_val(L, n);
            const double b = n2 < nl ? mg_smooth_val(L, n2) : 0.0;
            L.t[n] = a;
            if (n2 < nl) L.t[n2] = b;
          }
          if (!(ok = barrier())) break;
        }
      }
      if (!ok) break;
      coarse_gemv(F, nc, fcg_smem, gwarp, nwarps, lane);
      for (int l = M.L - 2; l >= 1; --l) {
        if (!(ok = barrier())) break;
        const MgLevel &L = M.lv[l];
        const double *ec = mg_e(M, l + 1);
        const int nyc = M.lv[l + 1].ny;
        const int64_t nl = (int64_t)L.nx * L.ny;
        for (int64_t n = gtid; n < nl; n += 2 * gth) {
          const int64_t n2 = n + gth;
          const double a = mg_post_val(L, ec, nyc, omega, n);
          const double b = n2 < nl ? mg_post_val(L, ec, nyc, omega, n2) : 0.0;
          L.t[n] = a;
          if (n2 < nl) L.t[n2] = b;
        }
      }
      if (!ok) break;
    } else if (F.coarse) {
      // (B) restriction
      for (int C = gwarp; C < nc; C += nwarps) {
        const int I = C / F.ncy, J = C % F.ncy;
        const int i0 = max(0, (I - 1) * F.cs + 1), i1 = min(F.nnx - 1, (I + 1) * F.cs - 1);
        const int j0 = max(0, (J - 1) * F.cs + 1), j1 = min(k.nny - 1, (J + 1) * F.cs - 1);
        const int ni = i1 - i0 + 1, nj = j1 - j0 + 1;
        const double inv = 1.0 / F.cs;
        double acc = 0.0;
        for (int e = lane; e < ni * nj; e += 32) {
          const int i = i0 + e / nj, j = j0 + e % nj;
          const double w = (1.0 - fabs((double)(i - I * F.cs)) * inv) * (1.0 - fabs((double)(j - J * F.cs)) * inv);
          acc = fma(w, (double)F.t[(int64_t)i * k.nny + j], acc);
        }
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) F.rc[C] = acc;
      }
      if (!(ok = barrier())) break;
      // (C) coarse solve
      coarse_gemv(F, nc, fcg_smem, gwarp, nwarps, lane);
      if (!(ok = barrier())) break;
      // (D) prolongation
      for (int c = blockIdx.x; c < nb; c += gridDim.x) {
        const int64_t n = (int64_t)c * kWide + threadIdx.x;
        if (n < nn && k.row_kind[n] >= 0) {
          const int i = (int)(n / k.nny), j = (int)(n % k.nny);
          const int I = i / F.cs, J = j / F.cs;
          const double fx = (double)(i - I * F.cs) / F.cs, fy = (double)(j - J * F.cs) / F.cs;
          const int I1 = min(I + 1, F.ncx - 1), J1 = min(J + 1, F.ncy - 1);
          double v = (1.0 - fx) * (1.0 - fy) * __ldcg(F.ec + I * F.ncy + J);
          v = fma(fx * (1.0 - fy), __ldcg(F.ec + I1 * F.ncy + J), v);
          v = fma((1.0 - fx) * fy, __ldcg(F.ec + I * F.ncy + J1), v);
          v = fma(fx * fy, __ldcg(F.ec + I1 * F.ncy + J1), v);
          F.zA[n] += (V)v;
        }
      }
    }
    if (!(ok = barrier())) break;
    if (M.L > 1) {
      // (E1) zA += P e_1 once per unknown node (Dirichlet nodes keep 0), so
      // that the post-smoothing reads it at its neighbours
      // two chunks a thread at a time: both nodes' loads are issued before
      // either store (the stores would otherwise hold back the next chunk's
      // loads, which the compiler cannot prove independent of them)
      const double *e1 = mg_e(M, 1);
      const int ny1 = M.lv[1].ny;
      for (int c = blockIdx.x; c < nb; c += 2 * gridDim.x) {
        const int64_t na = (int64_t)c * kWide + threadIdx.x, nb2 = na + (int64_t)gridDim.x * kWide;
        const bool ua = na < nn && k.row_kind[na] >= 0;
        const bool ub = nb2 < nn && k.row_kind[nb2] >= 0;
        double pa = 0.0, pb = 0.0, za = 0.0, zb = 0.0;
        if (ua) {
          const int i = (int)na / k.nny, j = (int)na - i * k.nny;  // the grid holds < 2^31 nodes
          pa = mg_prolong(e1, ny1, i, j);
          za = (double)F.zA[na];
        }
        if (ub) {
          const int i = (int)nb2 / k.nny, j = (int)nb2 - i * k.nny;
          pb = mg_prolong(e1, ny1, i, j);
          zb = (double)F.zA[nb2];
        }
        if (ua) F.zA[na] = (V)(za + pa);
        if (ub) F.zA[nb2] = (V)(zb + pb);
      }
      if (!(ok = barrier())) break;
    }
    // (E) post-smoothing and zF.Q_old (Q_old is this iteration's Ql)
    {
      double acc_zq = 0.0;
      for (int c = blockIdx.x; c < nb; c += gridDim.x) {
        const int64_t n = (int64_t)c * kWide + threadIdx.x;
        if (n < nn) {
          V zf = (V)0;
          if (k.row_kind[n] >= 0) {
            auto za = [&](int64_t m) { return F.zA[m]; };
            zf = vfma(om * F.dinv[n], r[n] - row_apply_v<V>(k, n, za), za(n));
          }
          F.zF[n] = zf;
          if (have_old) acc_zq = fma((double)zf, (double)Ql[n], acc_zq);
        }
      }
      double v[1] = {acc_zq}, o[1];
      cta_sum<1>(v, o);
      if (threadIdx.x == 0) F.part[3 * G + blockIdx.x] = o[0];
    }
    if (!(ok = barrier())) break;
    double beta = 0.0;
    if (have_old) {
      // its own region: phase F writes [0, 2 G) while slower CTAs may still read this
      double zq;
      final_sum_wide<1>(F.part + 3 * G, G, &zq);
      beta = -zq / pq_old;
    }
    // (F) P_new = zF + beta P_old at every neighbour (0 on Dirichlet nodes,
    // where zF and P_old are 0), Q_new = A P_new, p.q, p.r
    {
      const V bt = (V)beta;
      const bool ho = have_old;
      auto pnew = [&](int64_t m) { return ho ? vfma(bt, Pl[m], F.zF[m]) : F.zF[m]; };
      double acc[2] = {0.0, 0.0};
      for (int c = blockIdx.x; c < nb; c += gridDim.x) {
        const int64_t n = (int64_t)c * kWide + threadIdx.x;
        if (n < nn) {
          const V pv = pnew(n);
          const V qv = row_apply_v<V>(k, n, pnew);
          Pn[n] = pv;
          Qn[n] = qv;
          acc[0] = fma((double)pv, (double)qv, acc[0]);
          acc[1] = fma((double)pv, (double)r[n], acc[1]);
        }
      }
      double o[2];
      cta_sum<2>(acc, o);
      if (threadIdx.x == 0) {
        F.part[blockIdx.x] = o[0];
        F.part[G + blockIdx.x] = o[1];
      }
    }
    if (!(ok = barrier())) break;
    double pqpr[2];
    final_sum_wide<2>(F.part, G, pqpr);
    if (!(pqpr[0] > 0.0) || !(pqpr[1] == pqpr[1])) {
      ierr = 2;
      break;
    }
    alpha = pqpr[1] / pqpr[0];
    pq_old = pqpr[0];
    have_old = true;
    parity ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->iter = iter;
    S->rr = rr;
    S->best = best;
    S->best_iter = best_iter;
    S->ierr = ok ? ierr : 7;  // 7: a grid barrier timed out
    S->done = 1;
  }
}

// FP64 <-> FP32 helpers of the iterative refinement
__global__ void k_f64_to_f32(const double *__restrict__ a, float *__restrict__ b, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// x += e on unknown nodes (FP64 += FP32)
__global__ void k_add_f32(const int32_t *__restrict__ row_kind, const float *__restrict__ e, double *__restrict__ x,
                          int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && row_kind[i] >= 0) x[i] += (double)e[i];
}

__constant__ double c_ppr_reg[5][9];
// Patch layouts shared by many nodes (kind 3 + t): the relative offsets of
// the patch nodes in patch order and one pseudo-inverse for all of them.
constexpr int kPprTpl = 4, kPprTplMax = 25;
__constant__ int c_ppr_tpl_cnt[kPprTpl];
__constant__ int c_ppr_tpl_off[kPprTpl][kPprTplMax];
__constant__ double c_ppr_tpl_R[kPprTpl][5][kPprTplMax];

struct PprK {
  const double *phi, *h;
  const int32_t *kind, *ptr, *nodes;
  const double *rows;
  double *coef;  // [5][nn]
  double *efx, *efy;
  double2 *efxy;  // [nn] {efx, efy} (the FP64 push's gather)
  float *coef32;  // NULL, or [nn][8] FP32 records (mixed precision)
  int nny;
  int64_t nn;
};

// PPR: coef(2..6) = P_i * phi(patch_i) scaled by 1/h, 1/h^2; E = -grad.
__global__ void k_ppr(PprK k) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= k.nn) return;
  int kind = k.kind[n];
  double c[5] = {0, 0, 0, 0, 0};
  if (kind == 0) {
    double ph[9];
    const int64_t base = n - k.nny - 1;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) ph[3 * a + b] = k.phi[base + (int64_t)a * k.nny + b];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < 9; ++q) acc = fma(c_ppr_reg[r][q], ph[q], acc);
      c[r] = acc;
    }
  } else if (kind == 1) {
    int b0 = k.ptr[n], cnt = k.ptr[n + 1] - b0;
    const double *R = k.rows + 5 * (size_t)b0;
    for (int r = 0; r < 5; ++r) {
      double acc = 0.0;
      for (int q = 0; q < cnt; ++q) acc = fma(R[(size_t)r * cnt + q], k.phi[k.nodes[b0 + q]], acc);
      c[r] = acc;
    }
  } else if (kind >= 3) {
    // a shared layout: the patch's potentials first (all loads in flight),
    // then the rows, in patch order as for kind 1
    const int t = kind - 3, cnt = c_ppr_tpl_cnt[t];
    double ph[kPprTplMax];
#pragma unroll
    for (int q = 0; q < kPprTplMax; ++q) ph[q] = q < cnt ? k.phi[n + c_ppr_tpl_off[t][q]] : 0.0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < kPprTplMax; ++q)
        if (q < cnt) acc = fma(c_ppr_tpl_R[t][r][q], ph[q], acc);
      c[r] = acc;
    }
  }
  double h = k.h[n];
  if (kind != 2) {
    c[0] = c[0] / h;
    c[1] = c[1] / h;
    c[2] = c[2] / (h * h);
    c[3] = c[3] / (h * h);
    c[4] = c[4] / (h * h);
  }
  for (int r = 0; r < 5; ++r) k.coef[(size_t)r * k.nn + n] = c[r];
  k.efx[n] = -c[0];
  k.efy[n] = -c[1];
  k.efxy[n] = make_double2(-c[0], -c[1]);
  if (k.coef32) {  // mixed precision: one 32-byte FP32 record per node
    float4 *o = reinterpret_cast<float4 *>(k.coef32 + 8 * (size_t)n);
    o[0] = make_float4((float)-c[0], (float)-c[1], (float)c[0], (float)c[1]);
    o[1] = make_float4((float)c[2], (float)c[3], (float)c[4], 0.0f);
  }
}

// FP32 node records {efx, efy, c2, c3, c4, c5, c6, 0} from the FP64 fields
// (mixed precision, after the caller set a field).
__global__ void k_coef32(const double *__restrict__ efx, const double *__restrict__ efy,
                         const double *__restrict__ coef, float *__restrict__ coef32, int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  float4 *o = reinterpret_cast<float4 *>(coef32 + 8 * (size_t)n);
  o[0] = make_float4((float)efx[n], (float)efy[n], (float)coef[n], (float)coef[nn + n]);
  o[1] = make_float4((float)coef[2 * nn + n], (float)coef[3 * nn + n], (float)coef[4 * nn + n], 0.0f);
}

__global__ void k_efxy(const double *__restrict__ efx, const double *__restrict__ efy, double2 *__restrict__ efxy,
                       int64_t nn) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nn) efxy[n] = make_double2(efx[n], efy[n]);
}

__global__ void k_fill_u64(unsigned long long *a, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = 0ull;
}

// ----------------------------------------------------------------------------
// host helpers
// ----------------------------------------------------------------------------

static MeshK mesh_k() {
  MeshK m = g.m;
  m.xs = g.d_xs;
  m.ys = g.d_ys;
  m.element_index = g.d_element_index;
  m.node_index = g.d_node_index;
  m.elem_near = g.d_elem_near;
  return m;
}

template <class T>
static int dalloc(T **p, size_t n) {
  if (n == 0) n = 1;
  PIC_CUDA(cudaMalloc((void **)p, n * sizeof(T)));
  return PIC_OK;
}
template <class T>
static int upload(T **p, const T *h, size_t n) {
  int rc = dalloc(p, n);
  if (rc) return rc;
  if (h && n) PIC_CUDA(cudaMemcpy(*p, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return PIC_OK;
}

// Gauss-Jordan inverse with full pivoting of an n x n matrix (row-major),
// as BRINV does for the 6x6 normal matrix (PPR/BRINV.f90:11-70).
static bool brinv(double *a, int n) {
  std::vector<int> is(n), js(n);
  for (int k = 0; k < n; ++k) {
    double d = 0.0;
    for (int i = k; i < n; ++i)
      for (int j = k; j < n; ++j) {
        double p = std::fabs(a[i * n + j]);
        if (p > d) { d = p; is[k] = i; js[k] = j; }
      }
    if (d + 1.0 == 1.0) return false;
    if (is[k] != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[is[k] * n + j]);
    if (js[k] != k)
      for (int i = 0; i < n; ++i) std::swap(a[i * n + k], a[i * n + js[k]]);
    a[k * n + k] = 1.0 / a[k * n + k];
    for (int j = 0; j < n; ++j)
      if (j != k) a[k * n + j] = a[k * n + j] * a[k * n + k];
    for (int i = 0; i < n; ++i)
      if (i != k)
        for (int j = 0; j < n; ++j)
          if (j != k) a[i * n + j] = a[i * n + j] - a[i * n + k] * a[k * n + j];
    for (int i = 0; i < n; ++i)
      if (i != k) a[i * n + k] = -a[i * n + k] * a[k * n + k];
  }
  for (int k = n - 1; k >= 0; --k) {
    if (js[k] != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[js[k] * n + j]);
    if (is[k] != k)
      for (int i = 0; i < n; ++i) std::swap(a[i * n + k], a[i * n + is[k]]);
  }
  return true;
}

// Rows 2..6 of (A^T A)^-1 A^T for normalised patch offsets (GetEfield_SIDG_PPR.f90:158-197).
static bool ppr_rows(const std::vector<double> &px, const std::vector<double> &py, double *out5xn) {
  int n = (int)px.size();
  std::vector<double> AT(6 * n);
  for (int m = 0; m < n; ++m) {
    AT[0 * n + m] = 1.0;
    AT[1 * n + m] = px[m];
    AT[2 * n + m] = py[m];
    AT[3 * n + m] = px[m] * px[m];
    AT[4 * n + m] = px[m] * py[m];
    AT[5 * n + m] = py[m] * py[m];
  }
  double N[36];
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s = s + AT[a * n + m] * AT[b * n + m];
      N[a * 6 + b] = s;
    }
  if (!brinv(N, 6)) return false;
  for (int a = 1; a < 6; ++a)
    for (int m = 0; m < n; ++m) {
      double s = 0.0;
      for (int b = 0; b < 6; ++b) s = s + N[a * 6 + b] * AT[b * n + m];
      out5xn[(a - 1) * n + m] = s;
    }
  return true;
}

static void fcg_graphs_free();

static void free_all() {
  auto F = [](void *p) {
    if (p) cudaFree(p);
  };
  F(g.d_xs); F(g.d_ys); F(g.d_element_index); F(g.d_node_index); F(g.d_node_type); F(g.d_elem_near);
  F(g.d_phi_dir); F(g.d_cell_volume); F(g.d_rhs_fix); F(g.d_mass_q1); F(g.d_ife_mass); F(g.d_mass_rows);
  F(g.d_rf_nodes); F(g.d_rf_base);
  F(g.d_xt_ptr); F(g.d_xt_col); F(g.d_xt_val); F(g.d_row_kind); F(g.d_ex_cnt); F(g.d_ex_col);
  F(g.d_ex_val); F(g.d_ex_val32); F(g.d_fcg32); F(g.d_diag); F(g.d_ppr_kind); F(g.d_ppr_ptr); F(g.d_ppr_nodes); F(g.d_ppr_rows);
  F(g.d_ppr_h); F(g.d_phi); F(g.d_rho); F(g.d_efx); F(g.d_efy); F(g.d_efxy); F(g.d_coef); F(g.d_coef32); F(g.d_b); F(g.d_x);
  F(g.d_r); F(g.d_w); F(g.d_p[0]); F(g.d_p[1]); F(g.d_q); F(g.d_part); F(g.d_pcg); F(g.d_bar);
  F(g.d_z); F(g.d_dot); F(g.d_dot_ticket); F(g.d_fcg); F(g.d_fcg_P); F(g.d_fcg_Q); F(g.d_fcg_part);
  precond_free();
  diag_free();
  fcg_graphs_free();
  F(g.d_cell_count); F(g.d_cell_start); F(g.d_cell_fill); F(g.d_perm); F(g.d_perm2); F(g.d_sort_id);
  F(g.d_scan_blk); F(g.d_counters); F(g.d_hist); F(g.d_sel); F(g.d_cand); F(g.d_cand_slot);
  F(g.d_mcc_misc); F(g.d_mlist_key); F(g.d_mlist_slot); F(g.d_msel); F(g.d_ion_parent); F(g.d_ion_data); F(g.d_mcc_pslot); F(g.d_mcc_vel); F(g.d_ion_order);
  if (g.h_fcg) cudaFreeHost(g.h_fcg);
  for (int s = 0; s < PIC_MAX_SPECIES; ++s) {
    Species &p = g.sp[s];
    F(p.x); F(p.y); F(p.vx); F(p.vy); F(p.vz); F(p.loc); F(p.id);
    F(p.x2); F(p.y2); F(p.vx2); F(p.vy2); F(p.vz2); F(p.loc2); F(p.id2);
    F(p.q_acc); F(p.e_acc); F(p.rho_s); F(p.ek_s); F(p.ek_tot); F(p.prob);
  }
  if (g.ev0) cudaEventDestroy(g.ev0);
  if (g.ev1) cudaEventDestroy(g.ev1);
  if (g.st_copy) cudaStreamSynchronize(g.st_copy);
  for (auto &ev : g.step_ev)
    if (ev) cudaEventDestroy(ev);
  if (g.h_counters) cudaFreeHost(g.h_counters);
  for (auto &ev : g.ev_field)
    if (ev) cudaEventDestroy(ev);
  if (g.ev_copy_start) cudaEventDestroy(g.ev_copy_start);
  if (g.st_copy) cudaStreamDestroy(g.st_copy);
  if (g.st2) cudaStreamDestroy(g.st2);
  if (g.st) cudaStreamDestroy(g.st);
  g = Ctx();
}

int launch_locate(Species &s, int64_t begin, int64_t end) {
  if (end <= begin) return PIC_OK;
  k_locate<<<blocks_for(end - begin, 256), 256, 0, g.st>>>(mesh_k(), s.x, s.y, s.loc, begin, end,
                                                           g.d_counters + 1);
  PIC_LAUNCHED();
  return PIC_OK;
}

// Counters and zero fills on the library's stream go through kernels, not
// cudaMemcpyAsync / cudaMemsetAsync: copy-engine work of the stream queues
// behind a caller's field transfers in the same direction on the copy
// stream (pic_get_fields_async, ~0.6 ms for four 8 MB fields), and the
// stream's next step then starts only after them instead of alongside.
__global__ void k_counters_out(unsigned long long *dst, const unsigned long long *src, int n) {
  if ((int)threadIdx.x < n) dst[threadIdx.x] = src[threadIdx.x];
}

__global__ void k_zero(uint32_t *head, int nhead, uint4 *mid, int64_t nmid, uint32_t *tail, int ntail) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  if (t < nhead) head[t] = 0u;
  if (t < ntail) tail[t] = 0u;
  for (int64_t i = t; i < nmid; i += stride) mid[i] = make_uint4(0u, 0u, 0u, 0u);
}

int zero_async(void *p, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return PIC_OK;
  const uintptr_t a = (uintptr_t)p, e = a + bytes;
  if ((a | bytes) & 3u) {
    set_error("zero_async: pointer and size must be multiples of 4 bytes");
    return PIC_ERR_ARG;
  }
  uintptr_t m0 = (a + 15u) & ~(uintptr_t)15u, m1 = e & ~(uintptr_t)15u;
  if (m1 < m0) m0 = m1 = e;  // under 16 aligned bytes: all in the head
  const int nhead = (int)((m0 - a) / 4), ntail = (int)((e - m1) / 4);
  const int64_t nmid = (int64_t)((m1 - m0) / 16);
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((nmid + 255) / 256, 148 * 8));
  k_zero<<<(unsigned)blocks, 256, 0, st>>>((uint32_t *)a, nhead, (uint4 *)m0, nmid, (uint32_t *)m1, ntail);
  PIC_LAUNCHED();
  return PIC_OK;
}

// counters [first, first + n) (n <= 32) through the mapped mirror, one wait
static int read_counters(int first, int n, unsigned long long *v) {
  if (first < 0 || n < 0 || first + n > 32) {
    set_error("read_counters: counter range outside the 32 counters");
    return PIC_ERR_ARG;
  }
  k_counters_out<<<1, 32, 0, g.st>>>(g.hd_counters + first, g.d_counters + first, n);
  PIC_LAUNCHED();
  PIC_CUDA(cudaStreamSynchronize(g.st));
  const volatile unsigned long long *h = g.h_counters;
  for (int k = 0; k < n; ++k) v[k] = h[first + k];
  return PIC_OK;
}

static int read_counter(int idx, unsigned long long *v) { return read_counters(idx, 1, v); }

static int zero_counter(int idx) { return zero_async(g.d_counters + idx, sizeof(unsigned long long), g.st); }

// push and/or locate+deposit for one species
static int run_push(int sidx, bool do_push, bool do_deposit, bool do_energy) {
  Species &s = g.sp[sidx];
  if (s.n_slots == 0) return PIC_OK;
  FieldK f{g.d_efx, g.d_efy, g.d_coef, g.d_coef + g.nn, g.d_coef + 2 * g.nn, g.d_coef + 3 * g.nn,
           g.d_coef + 4 * g.nn, g.d_efxy};
  PushK prm;
  prm.qm = s.qm;
  prm.dt = g.P.dt;
  prm.mass = s.mass;
  prm.vref = g.v_ref;
  prm.do_push = do_push;
  prm.do_deposit = do_deposit;
  prm.do_energy = do_deposit && do_energy;
  for (int w = 0; w < 4; ++w) prm.wall[w] = g.P.wall_bc[w];
  SpK k{s.x, s.y, s.vx, s.vy, s.vz, s.loc, s.q_acc, s.e_acc, g.d_counters + 8 + sidx, g.d_counters + 1,
        s.n_slots, g.d_counters + 2};
  if (g.sel_push && do_deposit) k.sel = g.sel_sink[sidx];  // otherwise off (zero)
  if (s.f32) {
    const MeshK m = mesh_k();
    PushM pm;
    pm.qmdt = (float)(s.qm * g.P.dt);
    pm.dtx = (float)(g.P.dt / m.hx);
    pm.dty = (float)(g.P.dt / m.hy);
    pm.hx = (float)m.hx;
    pm.hy = (float)m.hy;
    pm.dt = g.P.dt;
    pm.hyd = m.hy;
    pm.inv_hy = 1.0 / m.hy;
    pm.mass = s.mass;
    pm.vref = g.v_ref;
    pm.do_push = do_push;
    pm.do_deposit = do_deposit;
    pm.do_energy = do_deposit && do_energy;
    for (int w = 0; w < 4; ++w) pm.wall[w] = g.P.wall_bc[w];
    if (g.push_bulk && g.push_stages) {
      // tiles bulk-copied by one thread (4 stages, 5 CTAs per SM)
      const int64_t ntiles = (s.n_slots + kPushTile - 1) / kPushTile;
      const unsigned grid = (unsigned)std::min<int64_t>(ntiles, g.push_grid);
      const size_t smem = 4 * sizeof(PushTile) + 4 * sizeof(uint64_t);
      if (g.axi)
        k_push_mixed_bulk<4, 5, true><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles,
                                                                       g.push_wait_limit, g.push_skip_copies);
      else
        k_push_mixed_bulk<4, 5, false><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles,
                                                                        g.push_wait_limit, g.push_skip_copies);
    } else if (g.axi) {
      // r-z: the default tiled form (4 stages, 5 CTAs per SM) or the direct one
      if (g.push_stages) {
        const int64_t ntiles = (s.n_slots + kPushTile - 1) / kPushTile;
        const unsigned grid = (unsigned)std::min<int64_t>(ntiles, g.push_grid);
        k_push_mixed_tiled<4, 5, true><<<grid, kPushTile, 4 * sizeof(PushTile), g.st>>>(m, g.d_coef32, pm, k, ntiles);
      } else {
        k_push_mixed<true><<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(m, g.d_coef32, pm, k);
      }
    } else if (g.push_stages) {
      const int64_t ntiles = (s.n_slots + kPushTile - 1) / kPushTile;
      const unsigned grid = (unsigned)std::min<int64_t>(ntiles, g.push_grid);
      const size_t smem = (size_t)g.push_stages * sizeof(PushTile);
      if (g.push_stages == 2)
        k_push_mixed_tiled<2><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles);
      else if (g.push_stages == 3)
        k_push_mixed_tiled<3><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles);
      else if (g.push_minb == 5)
        k_push_mixed_tiled<4, 5><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles);
      else if (g.push_minb == 6)
        k_push_mixed_tiled<4, 6><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles);
      else
        k_push_mixed_tiled<4><<<grid, kPushTile, smem, g.st>>>(m, g.d_coef32, pm, k, ntiles);
    } else {
      k_push_mixed<false><<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(m, g.d_coef32, pm, k);
    }
  } else if (g.push64_grid > 0 && g.push64_bulk) {
    const int64_t ntiles = (s.n_slots + kPushTile - 1) / kPushTile;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, g.push64_grid);
    const size_t smem = 3 * sizeof(PushTile64) + 3 * sizeof(uint64_t);
    if (g.axi)
      k_push_bulk<3, true><<<grid, kPushTile, smem, g.st>>>(mesh_k(), f, prm, k, ntiles, g.push_wait_limit,
                                                             g.push_skip_copies);
    else
      if (g.push64_minb == 5)
        k_push_bulk<3, false, 5><<<grid, kPushTile, smem, g.st>>>(mesh_k(), f, prm, k, ntiles, g.push_wait_limit,
                                                                   g.push_skip_copies);
      else
        k_push_bulk<3, false><<<grid, kPushTile, smem, g.st>>>(mesh_k(), f, prm, k, ntiles, g.push_wait_limit,
                                                                g.push_skip_copies);
  } else if (g.push64_grid > 0) {
    const int64_t ntiles = (s.n_slots + kPushTile - 1) / kPushTile;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, g.push64_grid);
    const size_t smem = 3 * sizeof(PushTile64);
    if (g.axi)
      k_push_tiled<3, true><<<grid, kPushTile, smem, g.st>>>(mesh_k(), f, prm, k, ntiles);
    else
      k_push_tiled<3, false><<<grid, kPushTile, smem, g.st>>>(mesh_k(), f, prm, k, ntiles);
  } else {
    if (g.axi)
      k_push<true><<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(mesh_k(), f, prm, k);
    else
      k_push<false><<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(mesh_k(), f, prm, k);
  }
  PIC_LAUNCHED();
  return PIC_OK;
}

// mixed precision: staging (FP64 absolute, set 2) <-> live (FP32 relative, set 1)
static int to_mixed(Species &s) {
  if (s.n_slots == 0) return PIC_OK;
  // the FP64 data sits in the live set; convert into set 2 and swap
  k_to_mixed<<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(
      mesh_k(), s.x, s.y, s.vx, s.vy, s.vz, s.loc, (float *)s.x2, (float *)s.y2, (float *)s.vx2, (float *)s.vy2,
      (float *)s.vz2, s.n_slots);
  PIC_LAUNCHED();
  std::swap(s.x, s.x2);
  std::swap(s.y, s.y2);
  std::swap(s.vx, s.vx2);
  std::swap(s.vy, s.vy2);
  std::swap(s.vz, s.vz2);
  return PIC_OK;
}

static int from_mixed(Species &s) {
  if (s.n_slots == 0) return PIC_OK;
  k_from_mixed<<<blocks_for(s.n_slots, 256), 256, 0, g.st>>>(
      mesh_k(), (const float *)s.x, (const float *)s.y, (const float *)s.vx, (const float *)s.vy,
      (const float *)s.vz, s.loc, s.x2, s.y2, s.vx2, s.vy2, s.vz2, s.n_slots);
  PIC_LAUNCHED();
  return PIC_OK;
}

static int zero_deposit(bool energy) {
  for (int s = 0; s < g.ns; ++s) {
    if (int rc = zero_async(g.sp[s].q_acc, g.nn * sizeof(unsigned long long), g.st)) return rc;
    if (energy)
      if (int rc = zero_async(g.sp[s].e_acc, g.nn * sizeof(unsigned long long), g.st)) return rc;
  }
  return PIC_OK;
}

static int run_rho(bool energy) {
  RhoK r;
  std::memset(&r, 0, sizeof r);
  r.ns = g.ns;
  r.energy = energy;
  r.L_ref = g.L_ref;
  r.n_ref = g.P.n_ref;
  r.axi = g.axi;
  for (int s = 0; s < g.ns; ++s) {
    r.q[s] = g.sp[s].q_acc;
    r.e[s] = g.sp[s].e_acc;
    r.rho_s[s] = g.sp[s].rho_s;
    r.ek_s[s] = g.sp[s].ek_s;
    r.ek_tot[s] = g.sp[s].ek_tot;
    r.wq[s] = g.sp[s].weight * g.sp[s].charge;
    r.w[s] = g.sp[s].weight;
  }
  k_rho<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(r, g.d_cell_volume, g.d_rho, g.nn);
  PIC_LAUNCHED();
  return PIC_OK;
}

static PcgK pcg_k(int parity) {
  PcgK k;
  k.row_kind = g.d_row_kind;
  k.ex_cnt = g.d_ex_cnt;
  k.ex_col = g.d_ex_col;
  k.ex_val = g.d_ex_val;
  k.ex_val32 = g.d_ex_val32;
  k.diag = g.d_diag;
  k.x = g.d_x;
  k.r = g.d_r;
  k.w = g.d_w;
  k.q = g.d_q;
  k.b = g.d_b;
  k.p_old = g.d_p[parity];
  k.p_new = g.d_p[parity ^ 1];
  k.part = g.d_part;
  k.st = g.d_pcg;
  k.phi = g.d_phi;
  k.node_type = g.d_node_type;
  k.nny = g.m.nny;
  k.n_mat = g.n_mat;
  k.nn = g.nn;
  k.nb = g.red_blocks;
  return k;
}

// Time-dependent wall potential: phi_D = base + value on the wall's nodes,
// written into the Dirichlet table the RHS reads and into phi.
__global__ void k_rf_set(const int32_t *__restrict__ nodes, const double *__restrict__ base, int count,
                         double value, double *__restrict__ phi_dir, double *__restrict__ phi) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int32_t n = nodes[k];
  const double v = base[k] + value;
  phi_dir[n] = v;
  phi[n] = v;
}

// IFE_Solve_2D.f90:104-121: bc_value(1) = V/Phi_ref*SIN(2*Pi*Frequency*time*time_ref)
// on the left Dirichlet boundary (there a commented-out line; here a switch,
// for either x wall): amplitude * sin(omega * time + phase).
static int rf_apply(double time) {
  if (g.rf_wall < 0 || g.rf_count == 0) return PIC_OK;
  const double value = g.rf_amp * std::sin(g.rf_omega * time + g.rf_phase);
  k_rf_set<<<(g.rf_count + 127) / 128, 128, 0, g.st>>>(g.d_rf_nodes, g.d_rf_base, g.rf_count, value, g.d_phi_dir,
                                                      g.d_phi);
  PIC_LAUNCHED();
  return PIC_OK;
}

static int run_rhs() {
  RhsK k;
  k.rho = g.d_rho;
  k.mass_q1 = g.d_mass_q1;
  k.ife_mass = g.d_ife_mass;
  k.mass_rows = g.d_mass_rows;
  k.rhs_fix = g.d_rhs_fix;
  k.phi_dir = g.d_phi_dir;
  k.xt_val = g.d_xt_val;
  k.node_type = g.d_node_type;
  k.element_index = g.d_element_index;
  k.xt_ptr = g.d_xt_ptr;
  k.xt_col = g.d_xt_col;
  k.b = g.d_b;
  k.nnx = g.m.nnx;
  k.nny = g.m.nny;
  k.ney = g.m.ney;
  k.nn = g.nn;
  k_rhs<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(k);
  PIC_LAUNCHED();
  return PIC_OK;
}

static int run_pcg(pic_solve_stats *stats) {
  PcgState h;
  std::memset(&h, 0, sizeof h);
  h.tol2 = g.P.pcg_tol * g.P.pcg_tol;
  h.maxit = g.P.pcg_maxit;
  PIC_CUDA(cudaMemcpyAsync(g.d_pcg, &h, sizeof h, cudaMemcpyHostToDevice, g.st));
  PcgK k0 = pcg_k(0);
  k_pcg_x0<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(k0);
  PIC_LAUNCHED();
  k_pcg_init<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k0);
  PIC_LAUNCHED();
  const int chunk = 32;
  int parity = 0;
  PcgState hs;
  if (g.coop_grid > 0) {
    PcgP P;
    P.k = pcg_k(0);
    P.p0 = g.d_p[0];
    P.p1 = g.d_p[1];
    P.partA = g.d_part;
    P.partB = g.d_part + g.red_blocks;
    P.bar = g.d_bar;
    P.bar_err = (int *)(g.d_bar + 2);
    P.spin_limit = g.pcg_spin_limit;
    P.bar_extra = g.pcg_bar_extra;
    if (int rc_ = zero_async(g.d_bar, 4 * sizeof(unsigned int), g.st)) return rc_;
    if (g.smem_grid > 0) {
      PcgS Q;
      Q.k = pcg_k(0);
      Q.w_g = g.d_p[1];  // strip exchange buffers: free while the smem solver runs
      Q.p_g = g.d_p[0];
      Q.partA = P.partA;
      Q.partB = P.partB;
      Q.bar = P.bar;
      Q.bar_err = P.bar_err;
      Q.spin_limit = P.spin_limit;
      Q.bar_extra = P.bar_extra;
      Q.H = g.m.nny + 1;
      void *args[] = {&Q};
      PIC_CUDA(cudaLaunchCooperativeKernel((const void *)k_pcg_smem, dim3(g.smem_grid), dim3(kWide), args,
                                           g.smem_bytes, g.st));
    } else {
      void *args[] = {&P};
      PIC_CUDA(cudaLaunchCooperativeKernel((const void *)k_pcg_persist, dim3(g.coop_grid), dim3(kWide),
                                           args, 0, g.st));
    }
    PIC_LAUNCHED();
    PIC_CUDA(cudaMemcpyAsync(&hs, g.d_pcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
    if (hs.ierr == 4) {
      set_error("pic_ife_solve: PCG grid barrier timed out");
      return PIC_ERR_CUDA;
    }
  }
  for (int it = 0; g.coop_grid == 0 && it < g.P.pcg_maxit + chunk; it += chunk) {
    for (int c = 0; c < chunk; ++c) {
      PcgK k = pcg_k(parity);
      k_pcg_dir<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k);
      PIC_LAUNCHED();
      k_pcg_upd<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k);
      PIC_LAUNCHED();
      parity ^= 1;
    }
    PIC_CUDA(cudaMemcpyAsync(&hs, g.d_pcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
    if (hs.done) break;
  }
  k_phi_out<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(g.d_x, g.d_node_type, g.d_phi_dir, g.d_phi, g.nn);
  PIC_LAUNCHED();
  if (stats) {
    stats->iterations = hs.iter;
    stats->ierr = hs.ierr;
    stats->rel_residual = (hs.normRHS > 0) ? std::sqrt(hs.normR / hs.normRHS) : 0.0;
    stats->fallback = 0;
    stats->outer = 0;
  }
  if (!(hs.normR == hs.normR)) {
    set_error("pic_ife_solve: NaN residual");
    return PIC_ERR_NAN;
  }
  if (hs.ierr == 1) {
    set_error("pic_ife_solve: PCG reached the iteration cap");
    return PIC_ERR_SOLVER_CAP;
  }
  if (hs.ierr >= 2) {
    set_error("pic_ife_solve: PCG breakdown");
    return PIC_ERR_BREAKDOWN;
  }
  return PIC_OK;
}

int launch_spmv(const double *v, double *out) {
  k_spmv<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(pcg_k(0), v, out);
  PIC_LAUNCHED();
  return PIC_OK;
}

// Preconditioner stage A: pre-smoothing and coarse correction into zA; with
// `learned`, also the learned stage's input t = r - A zA into d_pc_t.
static int precond_stage_a(const double *r, double *zA, int learned) {
  int rc;
  const int nb = blocks_for(g.nn, 256);
  const PcgK k0 = pcg_k(0);
  if (g.pc_sweeps > 0) {
    k_pc_pre<<<nb, 256, 0, g.st>>>(k0, r, g.d_pc_dinv, g.pc_omega, zA, g.d_pc_t);
    PIC_LAUNCHED();
    if (g.mg.L > 1 && (rc = mg_correct(g.d_pc_t, zA, 0))) return rc;
    if (g.pc_cs > 0 && (rc = coarse_correct(g.d_pc_t, zA, 0))) return rc;
  } else if (g.mg.L > 1) {
    if ((rc = mg_correct(r, zA, 1))) return rc;
  } else if (g.pc_cs > 0) {
    if ((rc = coarse_correct(r, zA, 1))) return rc;
  } else {
    if (int rc_ = zero_async(zA, g.nn * sizeof(double), g.st)) return rc_;
  }
  if (learned) {
    k_pc_mid<<<nb, 256, 0, g.st>>>(k0, r, zA, g.d_pc_t);
    PIC_LAUNCHED();
  }
  return PIC_OK;
}

// Preconditioner stage B: zF = post-smoothing of zA (+ the learned stage's
// y); inside FCG (fk != NULL) also the A-orthogonalisation coefficients.
static int precond_stage_b(const double *r, const double *zA, double *zF, int learned, const FcgK *fk) {
  FcgK k{};
  if (fk) {
    k = *fk;
  } else {
    k.op = pcg_k(0);
    k.part = g.d_part;
    k.ring = 1;
    k.window = 1;
  }
  const int smooth = (g.pc_sweeps > 0 && (coarse_on() || learned)) ? 1 : 0;
  k_fcg_post<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k, r, zA, learned ? g.d_pc_y : nullptr, g.d_pc_dinv,
                                                         g.pc_omega, smooth, zF);
  PIC_LAUNCHED();
  return PIC_OK;
}

// z = M(r) (full != 0) or the classical stages only (full == 0).  Returns 1
// when the learned stage's callback fails, a negative PIC_ERR_* on a CUDA
// error.
int precond_apply(int full, const double *r, double *z) {
  int rc;
  if ((rc = precond_prepare())) return rc;
  if (!full) return precond_stage_a(r, z, 0);
  const int learned = precond_learned_on();
  if ((rc = precond_stage_a(r, g.d_pc_za, learned))) return rc;
  if (learned && precond_callback()) return 1;
  return precond_stage_b(r, g.d_pc_za, z, learned, nullptr);
}

static int dot2(const double *a, const double *b, const double *c, const double *d, double out[2]) {
  DotK k{a, b, c, d, g.d_part, g.d_dot, g.d_dot_ticket, g.nn, g.red_blocks};
  k_dot<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k);
  PIC_LAUNCHED();
  PIC_CUDA(cudaMemcpyAsync(out, g.d_dot, 2 * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  return PIC_OK;
}

static void fcg_graphs_free() {
  for (auto &e : g.fcg_graph)
    if (e) {
      cudaGraphExecDestroy(e);
      e = nullptr;
    }
  g.fcg_graph_key = 0;
}

// Captures `body` (kernel launches on g.st) into an executable graph and
// records how many kernels it launches.
template <class F>
static int fcg_capture(cudaGraphExec_t *ex, long long *launches, F body) {
  cudaGraph_t gr = nullptr;
  const long long before = g_launches;
  PIC_CUDA(cudaStreamBeginCapture(g.st, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  const cudaError_t e = cudaStreamEndCapture(g.st, &gr);
  *launches = g_launches - before;
  g_launches = before;
  if (rc) {
    if (gr) cudaGraphDestroy(gr);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  const cudaError_t ei = cudaGraphInstantiate(ex, gr, 0);
  cudaGraphDestroy(gr);
  if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
  return PIC_OK;
}

static int fcg_graph_launch(int i) {
  PIC_CUDA(cudaGraphLaunch(g.fcg_graph[i], g.st));
  g_launches += g.fcg_graph_launches[i];
  return PIC_OK;
}

static int fcg_alloc() {
  if (g.d_fcg_P) return PIC_OK;
  int rc;
  const size_t ring = (size_t)(PIC_FCG_MAX_WINDOW + 1) * (size_t)g.nn;
  if ((rc = dalloc(&g.d_fcg_P, ring))) return rc;
  if ((rc = dalloc(&g.d_fcg_Q, ring))) return rc;
  if ((rc = dalloc(&g.d_fcg_part, (size_t)PIC_FCG_MAX_WINDOW * g.red_blocks))) return rc;
  return PIC_OK;
}

// Flexible CG with the registered preconditioner.  Iterations are enqueued
// in chunks sized from the previous solve's count; kernels after convergence
// inside a chunk return at once.  Convergence is accepted only on the true
// residual b - A x (recomputed in FP64 with the same operator and canonical
// dots); if the recursive residual drifted, the iteration restarts from the
// true one with no previous directions.  Returns 0 when converged, else the
// reason it hands over to Jacobi-PCG (the fallback codes of pic_solve_stats).
// The FP64 FCG as one cooperative kernel between two k_fcg_resid launches:
// the initial residual and its norms, the iterations, the true residual of
// the result.  The host writes the state's fixed fields from pinned memory
// and reads the state back once, after the judge (one wait per solve,
// three kernels).  Returns as run_fcg: 0 converged, else the fallback code.
static int run_fcg_persist64(pic_solve_stats *stats, int *fcg_iters, int *rc_out) {
  const int64_t nn = g.nn;
  int rc;
  if (!g.h_fcg) PIC_CUDA(cudaMallocHost(&g.h_fcg, sizeof(FcgState)));
  FcgState &hs = *static_cast<FcgState *>(g.h_fcg);
  std::memset(&hs, 0, sizeof hs);
  hs.tol2 = g.P.pcg_tol * g.P.pcg_tol;
  hs.maxit = std::min(g.P.pcg_maxit, 1000);
  hs.stall_window = 50;
  PcgK k0 = pcg_k(0);
  PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &hs, sizeof hs, cudaMemcpyHostToDevice, g.st));
  k_fcg_resid<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k0, g.d_dot_ticket, g.d_fcg, 1);
  PIC_LAUNCHED();
  FcgP<double> F;
  F.k = k0;
  F.part = g.d_fcg_part;
  F.ainv = g.d_pc_ainv;
  F.ainv_scale = g.pc_ainv_scale;
  F.ainv_ld = g.pc_ainv_ld;
  F.rc = g.d_pc_rc;
  F.ec = g.d_pc_ec;
  F.nnx = g.m.nnx;
  F.cs = g.pc_cs;
  F.ncx = g.pc_ncx;
  F.ncy = g.pc_ncy;
  F.coarse = g.pc_cs > 0 ? 1 : 0;
  F.mg = g.mg;
  if (g.mg.L > 1) {  // the coarsest level's r and z feed the dense solve
    const MgLevel &C = g.mg.lv[g.mg.L - 1];
    F.rc = C.r;
    F.ec = C.z;
    F.ncx = C.nx;
    F.ncy = C.ny;
  }
  F.omega = g.pc_omega;
  F.s = g.d_fcg;
  F.bar = g.d_bar;
  F.bar_err = (int *)(g.d_bar + 2);
  F.spin_limit = g.pcg_spin_limit;
  F.bar_extra = g.pcg_bar_extra;
  F.x = g.d_x;
  F.r = g.d_r;
  F.r2 = g.d_w;  // free while FCG runs
  F.dinv = g.d_pc_dinv;
  F.zA = g.d_pc_za;
  F.t = g.d_pc_t;
  F.zF = g.d_z;
  F.P0 = g.d_fcg_P;
  F.P1 = g.d_fcg_P + nn;
  F.Q0 = g.d_fcg_Q;
  F.Q1 = g.d_fcg_Q + nn;
  const void *fn = (const void *)k_fcg_persist<double>;
  const size_t smem = (size_t)g.pc_ainv_ld * sizeof(double);  // coarse_gemv's staging
  if (!g.fcg_smem_set || g.fcg_smem_set != smem) {
    PIC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    g.fcg_smem_set = smem;
  }
  auto finish = [&](int fallback) {
    *fcg_iters = hs.iter;
    if (stats) {
      stats->iterations = hs.iter;
      stats->rel_residual = hs.rhs > 0 ? std::sqrt(hs.rr / hs.rhs) : 0.0;
      stats->ierr = 0;
    }
    if (!fallback) g.fcg_last_iters = std::max(hs.iter, 1);
    return fallback;
  };
  for (int judged = 0;; ++judged) {
    if (int rc_ = zero_async(g.d_bar, 4 * sizeof(unsigned int), g.st)) return rc_;
    void *args[] = {&F};
    PIC_CUDA(cudaLaunchCooperativeKernel(fn, dim3(g.fcg_coop_grid), dim3(kWide), args, smem, g.st));
    PIC_LAUNCHED();
    // the judge: the true residual of the result (r is the next start)
    k_fcg_resid<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(k0, g.d_dot_ticket, g.d_fcg, 0);
    PIC_LAUNCHED();
    PIC_CUDA(cudaMemcpyAsync(&hs, g.d_fcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
    if (hs.ierr == 7) {
      set_error("pic_ife_solve: FCG grid barrier timed out");
      *rc_out = PIC_ERR_CUDA;
      return 1;
    }
    if (hs.ierr) return finish(hs.ierr);
    if (!(hs.rhs > 0.0) || hs.rr / hs.rhs <= hs.tol2) return finish(0);
    if (judged >= 3 || hs.iter >= hs.maxit) return finish(6);
    hs.done = 0;
    hs.count = 0;
    PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &hs, sizeof hs, cudaMemcpyHostToDevice, g.st));
  }
  (void)rc;
}

static int run_fcg(pic_solve_stats *stats, int *fcg_iters, int *rc_out) {
  *rc_out = PIC_OK;
  const int64_t nn = g.nn;
  const int nb = blocks_for(nn, 256);
  int rc;
  if ((rc = fcg_alloc())) { *rc_out = rc; return 1; }
  if (g.fcg_coop_grid > 0 && g.fcg_window == 1 && g.pc_sweeps > 0 && !(g.mixed && g.fcg_inner32) &&
      g.fcg_fused) {
    if ((rc = precond_prepare())) { *rc_out = rc; return 1; }
    if (!precond_learned_on()) return run_fcg_persist64(stats, fcg_iters, rc_out);
  }
  PcgK k0 = pcg_k(0);
  k0.w = g.d_z;
  FcgK fk{k0, g.d_fcg_P, g.d_fcg_Q, g.d_fcg_part, g.d_fcg, 0, g.fcg_window + 1, g.fcg_window};
  k_pcg_x0<<<nb, 256, 0, g.st>>>(k0);
  PIC_LAUNCHED();
  k_spmv<<<nb, 256, 0, g.st>>>(k0, g.d_x, g.d_q);
  PIC_LAUNCHED();
  k_fcg_r0<<<nb, 256, 0, g.st>>>(g.d_row_kind, g.d_b, g.d_q, g.d_r, nn);
  PIC_LAUNCHED();
  double s2[2];
  if ((rc = dot2(g.d_b, g.d_b, g.d_r, g.d_r, s2))) { *rc_out = rc; return 1; }
  FcgState hs{};
  hs.rhs = s2[0];
  hs.rr = s2[1];
  hs.best = s2[1];
  hs.tol2 = g.P.pcg_tol * g.P.pcg_tol;
  hs.maxit = std::min(g.P.pcg_maxit, 1000);
  hs.stall_window = 50;
  hs.count = 0;
  auto finish = [&](int fallback) {
    *fcg_iters = hs.iter;
    if (stats) {
      stats->iterations = hs.iter;
      stats->rel_residual = hs.rhs > 0 ? std::sqrt(hs.rr / hs.rhs) : 0.0;
      stats->ierr = 0;
    }
    if (!fallback) g.fcg_last_iters = std::max(hs.iter, 1);
    return fallback;
  };
  if (!(hs.rhs > 0.0) || hs.rr / hs.rhs <= hs.tol2) return finish(0);
  PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &hs, sizeof hs, cudaMemcpyHostToDevice, g.st));
  // stage buffers exist before any capture; graphs are rebuilt when the
  // stage configuration or the window changed
  if ((rc = precond_prepare())) { *rc_out = rc; return 1; }
  const int learned = precond_learned_on();
  const bool use_graphs = g.fcg_graphs != 0;
  if (use_graphs) {
    unsigned long long key = g.fcg_graph_gen;
    key = key * 1000003ull + (unsigned long long)g.fcg_window;
    key = key * 1000003ull + (unsigned long long)(g.pc_sweeps * 2 + learned);
    key = key * 1000003ull + (unsigned long long)g.pc_cs;
    key = key * 1000003ull + (unsigned long long)g.mg.L;
    key = key * 1000003ull + (unsigned long long)std::llround(g.pc_omega * 1e9);
    if (key != g.fcg_graph_key) {
      fcg_graphs_free();
      g.fcg_graph_key = key;
    }
  }
  int judged = 0;
  if (g.fcg_coop_grid > 0 && g.fcg_window == 1 && !learned && g.pc_sweeps > 0) {
    auto common = [&](auto &F) {
      F.k = k0;
      F.part = g.d_fcg_part;
      F.ainv = g.d_pc_ainv;
      F.ainv_scale = g.pc_ainv_scale;
      F.ainv_ld = g.pc_ainv_ld;
      F.rc = g.d_pc_rc;
      F.ec = g.d_pc_ec;
      F.nnx = g.m.nnx;
      F.cs = g.pc_cs;
      F.ncx = g.pc_ncx;
      F.ncy = g.pc_ncy;
      F.coarse = g.pc_cs > 0 ? 1 : 0;
      F.mg = g.mg;
      if (g.mg.L > 1) {  // the coarsest level's r and z feed the dense solve
        const MgLevel &C = g.mg.lv[g.mg.L - 1];
        F.rc = C.r;
        F.ec = C.z;
        F.ncx = C.nx;
        F.ncy = C.ny;
      }
      F.omega = g.pc_omega;
      F.s = g.d_fcg;
      F.bar = g.d_bar;
      F.bar_err = (int *)(g.d_bar + 2);
      F.spin_limit = g.pcg_spin_limit;
      F.bar_extra = g.pcg_bar_extra;
    };
    auto launch = [&](auto &F, const void *fn) -> int {
      if (int rc_ = zero_async(g.d_bar, 4 * sizeof(unsigned int), g.st)) return rc_;
      void *args[] = {&F};
      const size_t smem = (size_t)g.pc_ainv_ld * sizeof(double);  // coarse_gemv's staging
      PIC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PIC_CUDA(cudaLaunchCooperativeKernel(fn, dim3(g.fcg_coop_grid), dim3(kWide), args, smem, g.st));
      PIC_LAUNCHED();
      return PIC_OK;
    };
    auto true_residual = [&]() -> int {
      k_spmv<<<nb, 256, 0, g.st>>>(k0, g.d_x, g.d_q);
      PIC_LAUNCHED();
      k_fcg_r0<<<nb, 256, 0, g.st>>>(g.d_row_kind, g.d_b, g.d_q, g.d_r, nn);
      PIC_LAUNCHED();
      int r2 = dot2(g.d_r, g.d_r, nullptr, nullptr, s2);
      if (!r2) hs.rr = s2[0];
      return r2;
    };
    if (g.mixed && g.fcg_inner32) {
      // Mixed precision: FP32 inner FCG solves of A e = r inside FP64 iterative
      // refinement (x += e, r = b - A x in FP64, tested against the tolerance).
      if (!g.d_fcg32) {
        if ((rc = dalloc(&g.d_fcg32, 11 * (size_t)nn))) { *rc_out = rc; return 1; }
        k_f64_to_f32<<<nb, 256, 0, g.st>>>(g.d_pc_dinv, g.d_fcg32 + 10 * (size_t)nn, nn);
        PIC_LAUNCHED();
      }
      float *v32 = g.d_fcg32;
      FcgP<float> F;
      common(F);
      F.r = v32;
      F.r2 = v32 + nn;
      F.x = v32 + 2 * nn;
      F.zA = v32 + 3 * nn;
      F.t = v32 + 4 * nn;
      F.zF = v32 + 5 * nn;
      F.P0 = v32 + 6 * nn;
      F.P1 = v32 + 7 * nn;
      F.Q0 = v32 + 8 * nn;
      F.Q1 = v32 + 9 * nn;
      F.dinv = v32 + 10 * nn;
      int outer = 0, total = 0;
      for (;;) {
        if (hs.rr / hs.rhs <= hs.tol2) {
          hs.iter = total;
          if (stats) stats->outer = outer;
          return finish(0);
        }
        if (++outer > 8 || total >= hs.maxit) {
          hs.iter = total;
          if (stats) stats->outer = outer;
          return finish(6);
        }
        k_f64_to_f32<<<nb, 256, 0, g.st>>>(g.d_r, F.r, nn);
        PIC_LAUNCHED();
        if (int rc_ = zero_async(F.x, nn * sizeof(float), g.st)) return rc_;
        FcgState in{};
        in.rhs = hs.rr;
        in.rr = hs.rr;
        in.best = hs.rr;
        // the reduction the outer residual still needs, but at most 1e-5 per
        // sweep (FP32 vectors: a 1e-6 target costs more iterations than the
        // extra sweep it saves)
        in.tol2 = std::max(hs.tol2 * hs.rhs / hs.rr, 1e-10);
        in.maxit = hs.maxit - total;
        in.stall_window = 50;
        PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &in, sizeof in, cudaMemcpyHostToDevice, g.st));
        if ((rc = launch(F, (const void *)k_fcg_persist<float>))) { *rc_out = rc; return 1; }
        PIC_CUDA(cudaMemcpyAsync(&in, g.d_fcg, sizeof in, cudaMemcpyDeviceToHost, g.st));
        PIC_CUDA(cudaStreamSynchronize(g.st));
        if (in.ierr == 7) {
          set_error("pic_ife_solve: FCG grid barrier timed out");
          *rc_out = PIC_ERR_CUDA;
          return 1;
        }
        total += in.iter;
        const double rr_before = hs.rr;
        k_add_f32<<<nb, 256, 0, g.st>>>(g.d_row_kind, F.x, g.d_x, nn);
        PIC_LAUNCHED();
        if ((rc = true_residual())) { *rc_out = rc; return 1; }
        if (in.ierr && !(hs.rr < 0.25 * rr_before)) {  // the sweep failed and gained little
          hs.iter = total;
          if (stats) stats->outer = outer;
          return finish(in.ierr);
        }
      }
    }
    FcgP<double> F;
    common(F);
    F.x = g.d_x;
    F.r = g.d_r;
    F.r2 = g.d_w;  // free while FCG runs
    F.dinv = g.d_pc_dinv;
    F.zA = g.d_pc_za;
    F.t = g.d_pc_t;
    F.zF = g.d_z;
    F.P0 = g.d_fcg_P;
    F.P1 = g.d_fcg_P + nn;
    F.Q0 = g.d_fcg_Q;
    F.Q1 = g.d_fcg_Q + nn;
    for (;;) {
      if ((rc = launch(F, (const void *)k_fcg_persist<double>))) { *rc_out = rc; return 1; }
      PIC_CUDA(cudaMemcpyAsync(&hs, g.d_fcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
      PIC_CUDA(cudaStreamSynchronize(g.st));
      if (hs.ierr == 7) {
        set_error("pic_ife_solve: FCG grid barrier timed out");
        *rc_out = PIC_ERR_CUDA;
        return 1;
      }
      if (hs.ierr) return finish(hs.ierr);
      if ((rc = true_residual())) { *rc_out = rc; return 1; }
      if (hs.rr / hs.rhs <= hs.tol2) return finish(0);
      if (++judged > 3 || hs.iter >= hs.maxit) return finish(6);
      hs.done = 0;
      hs.count = 0;
      PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &hs, sizeof hs, cudaMemcpyHostToDevice, g.st));
    }
  }
  int64_t enq = 0;  // iterations enqueued (ring slot = enq mod m)
  for (;;) {
    int chunk = g.fcg_last_iters - hs.iter;
    chunk = std::min(std::max(chunk, 2), 64);
    for (int c = 0; c < chunk; ++c) {
      ++g.fcg_precond_calls;
      const int slot = (int)(enq++ % (g.fcg_window + 1));
      if (use_graphs) {
        if (!g.fcg_graph[0] && (rc = fcg_capture(&g.fcg_graph[0], &g.fcg_graph_launches[0],
                                                 [&] { return precond_stage_a(g.d_r, g.d_pc_za, learned); }))) {
          *rc_out = rc;
          return 1;
        }
        if ((rc = fcg_graph_launch(0))) { *rc_out = rc; return 1; }
      } else if ((rc = precond_stage_a(g.d_r, g.d_pc_za, learned))) {
        *rc_out = rc;
        return 1;
      }
      if (learned && precond_callback()) {
        PIC_CUDA(cudaMemcpyAsync(&hs, g.d_fcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
        PIC_CUDA(cudaStreamSynchronize(g.st));
        return finish(5);
      }
      fk.slot = slot;
      auto tail = [&] {
        int r2;
        if ((r2 = precond_stage_b(g.d_r, g.d_pc_za, g.d_z, learned, &fk))) return r2;
        k_fcg_dir<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(fk);
        PIC_LAUNCHED();
        k_fcg_upd<<<g.red_blocks, PIC_RED_THREADS, 0, g.st>>>(fk);
        PIC_LAUNCHED();
        return PIC_OK;
      };
      if (use_graphs) {
        if (!g.fcg_graph[1 + slot] &&
            (rc = fcg_capture(&g.fcg_graph[1 + slot], &g.fcg_graph_launches[1 + slot], tail))) {
          *rc_out = rc;
          return 1;
        }
        if ((rc = fcg_graph_launch(1 + slot))) { *rc_out = rc; return 1; }
      } else if ((rc = tail())) {
        *rc_out = rc;
        return 1;
      }
    }
    PIC_CUDA(cudaMemcpyAsync(&hs, g.d_fcg, sizeof hs, cudaMemcpyDeviceToHost, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
    if (!hs.done) continue;
    if (hs.ierr) return finish(hs.ierr);
    // judge the converged iterate on its true residual
    k_spmv<<<nb, 256, 0, g.st>>>(k0, g.d_x, g.d_q);
    PIC_LAUNCHED();
    k_fcg_r0<<<nb, 256, 0, g.st>>>(g.d_row_kind, g.d_b, g.d_q, g.d_r, nn);
    PIC_LAUNCHED();
    if ((rc = dot2(g.d_r, g.d_r, nullptr, nullptr, s2))) { *rc_out = rc; return 1; }
    hs.rr = s2[0];
    if (hs.rr / hs.rhs <= hs.tol2) return finish(0);
    if (++judged > 3 || hs.iter >= hs.maxit) return finish(6);
    hs.done = 0;
    hs.count = 0;
    PIC_CUDA(cudaMemcpyAsync(g.d_fcg, &hs, sizeof hs, cudaMemcpyHostToDevice, g.st));
  }
}

// Solver dispatch: flexible CG with the registered preconditioner, else (or
// after an FCG hand-over) Jacobi-PCG warm-started from the FCG iterate.
static int run_solve(pic_solve_stats *stats) {
  if (g.solver == PIC_SOLVER_FCG_UNET && ((g.pc_learned && g.precond) || coarse_on() || g.pc_sweeps > 0)) {
    int fcg_iters = 0, rc = PIC_OK;
    if (stats) stats->outer = 0;
    int fallback = run_fcg(stats, &fcg_iters, &rc);
    if (rc) return rc;
    k_phi_out<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(g.d_x, g.d_node_type, g.d_phi_dir, g.d_phi, g.nn);
    PIC_LAUNCHED();
    if (!fallback) {
      if (stats) stats->fallback = 0;
      return PIC_OK;
    }
    int prc = run_pcg(stats);
    if (stats) {
      stats->iterations += fcg_iters;
      stats->fallback = fallback;
    }
    return prc;
  }
  return run_pcg(stats);
}

static int run_ppr(cudaStream_t stream = nullptr) {
  PprK k;
  k.phi = g.d_phi;
  k.h = g.d_ppr_h;
  k.kind = g.d_ppr_kind;
  k.ptr = g.d_ppr_ptr;
  k.nodes = g.d_ppr_nodes;
  k.rows = g.d_ppr_rows;
  k.coef = g.d_coef;
  k.efx = g.d_efx;
  k.efy = g.d_efy;
  k.efxy = g.d_efxy;
  k.coef32 = g.d_coef32;
  k.nny = g.m.nny;
  k.nn = g.nn;
  k_ppr<<<blocks_for(g.nn, 256), 256, 0, stream ? stream : g.st>>>(k);
  PIC_LAUNCHED();
  return PIC_OK;
}

// The library's stream waits for the copies of pic_get_fields_async (still
// reading the fields) and pic_set_field_async (still writing them) queued
// for the fields in `mask` (bit f: 0 rho, 1 phi, 2 efx, 3 efy), before
// anything that writes, or after an upload reads, them.
int fields_fence(unsigned mask) {
  for (int f = 0; f < 4; ++f)
    if (g.copy_pending & mask & (1u << f)) PIC_CUDA(cudaStreamWaitEvent(g.st, g.ev_field[f], 0));
  return PIC_OK;
}

static int check_init() {
  if (!g.inited) {
    set_error("library not initialised (pic_init)");
    return PIC_ERR_STATE;
  }
  return PIC_OK;
}

static int check_species(int s) {
  if (s < 0 || s >= g.ns) {
    set_error("species index out of range");
    return PIC_ERR_ARG;
  }
  return PIC_OK;
}

}  // namespace pic

using namespace pic;

extern "C" {

const char *pic_last_error(void) { return g_err.c_str(); }
int64_t pic_kernel_launches(void) { return (int64_t)g_launches; }

int pic_set_preconditioner(pic_precond_fn fn, void *user) {
  g.precond = fn;
  g.precond_user = user;
  return PIC_OK;
}

int pic_set_solver(int32_t solver) {
  if (solver != PIC_SOLVER_JPCG && solver != PIC_SOLVER_FCG_UNET) {
    set_error("pic_set_solver: unknown solver");
    return PIC_ERR_ARG;
  }
  g.solver = solver;
  return PIC_OK;
}

int pic_set_fcg_window(int32_t window) {
  if (window < 1 || window > PIC_FCG_MAX_WINDOW) {
    set_error("pic_set_fcg_window: window must be 1..8");
    return PIC_ERR_ARG;
  }
  g.fcg_window = window;
  return PIC_OK;
}

int pic_set_precond_stages(int32_t smoothing, double omega, int32_t learned) {
  if (smoothing < 0 || smoothing > 1 || !(omega > 0.0 && omega < 2.0)) {
    set_error("pic_set_precond_stages: smoothing must be 0 or 1 and 0 < omega < 2");
    return PIC_ERR_ARG;
  }
  g.pc_sweeps = smoothing;
  g.pc_omega = omega;
  g.pc_learned = learned ? 1 : 0;
  return PIC_OK;
}

int pic_coarse_setup(const pic_mesh_desc *mesh, int32_t coarse_cells) {
  if (!g.inited) {
    set_error("pic_coarse_setup: library not initialised");
    return PIC_ERR_STATE;
  }
  if (!mesh || mesh->nnx != g.m.nnx || mesh->nny != g.m.nny) {
    set_error("pic_coarse_setup: mesh does not match the initialised one");
    return PIC_ERR_ARG;
  }
  return coarse_setup(mesh, coarse_cells);
}

int pic_multigrid_setup(const pic_mesh_desc *mesh, int32_t max_coarse_nodes) {
  if (!g.inited) {
    set_error("pic_multigrid_setup: library not initialised (pic_init)");
    return PIC_ERR_STATE;
  }
  if (!mesh || mesh->nnx != g.m.nnx || mesh->nny != g.m.nny) {
    set_error("pic_multigrid_setup: mesh does not match the initialised one");
    return PIC_ERR_ARG;
  }
  if (max_coarse_nodes > 9000) {
    set_error("pic_multigrid_setup: max_coarse_nodes above 9000");
    return PIC_ERR_ARG;
  }
  return mg_setup(mesh, max_coarse_nodes);
}

int pic_precond_apply(int32_t full, const double *r_dev, double *z_dev) {
  if (!g.inited) {
    set_error("pic_precond_apply: library not initialised");
    return PIC_ERR_STATE;
  }
  if (!r_dev || !z_dev) {
    set_error("pic_precond_apply: null vector");
    return PIC_ERR_ARG;
  }
  int rc = precond_apply(full, r_dev, z_dev);
  if (rc > 0) {
    set_error("pic_precond_apply: the learned correction failed");
    return PIC_ERR_STATE;
  }
  return rc;
}

int pic_set_fcg_inner(int32_t fp32) {
  if (fp32 != 0 && fp32 != 1) {
    set_error("pic_set_fcg_inner: 0 (FP64 iterations) or 1 (FP32 iterations in FP64 refinement)");
    return PIC_ERR_ARG;
  }
  g.fcg_inner32 = fp32;
  return PIC_OK;
}

int pic_cuda_stream(void **stream) {
  if (!g.inited) {
    set_error("pic_cuda_stream: library not initialised");
    return PIC_ERR_STATE;
  }
  if (stream) *stream = (void *)g.st;
  return PIC_OK;
}

int pic_apply_operator(const double *v_dev, double *out_dev) {
  if (!g.inited) {
    set_error("pic_apply_operator: library not initialised");
    return PIC_ERR_STATE;
  }
  if (!v_dev || !out_dev) {
    set_error("pic_apply_operator: null vector");
    return PIC_ERR_ARG;
  }
  k_spmv<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(pcg_k(0), v_dev, out_dev);
  PIC_LAUNCHED();
  return PIC_OK;
}

int pic_solver_vectors(double **b_dev, double **phi_dev) {
  if (!g.inited) {
    set_error("pic_solver_vectors: library not initialised");
    return PIC_ERR_STATE;
  }
  if (b_dev) *b_dev = g.d_b;
  if (phi_dev) *phi_dev = g.d_phi;
  return PIC_OK;
}

int pic_device_timer(int32_t op, double *ms_out) {
  if (!g.inited) {
    set_error("pic_device_timer: library not initialised");
    return PIC_ERR_STATE;
  }
  static cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (!t0) {
    PIC_CUDA(cudaEventCreate(&t0));
    PIC_CUDA(cudaEventCreate(&t1));
  }
  if (op == 0) {
    PIC_CUDA(cudaEventRecord(t0, g.st));
    return PIC_OK;
  }
  if (op != 1) return PIC_ERR_ARG;
  PIC_CUDA(cudaEventRecord(t1, g.st));
  PIC_CUDA(cudaEventSynchronize(t1));
  float ms = 0;
  PIC_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  if (ms_out) *ms_out = ms;
  return PIC_OK;
}

void pic_finalize(void) {
  if (g.inited) cudaStreamSynchronize(g.st);
  free_all();
}

int pic_init(const pic_mesh_desc *mesh, const pic_params *params) {
  if (!mesh || !params) {
    set_error("pic_init: null argument");
    return PIC_ERR_ARG;
  }
  if (g.inited) free_all();
  const pic_params &P = *params;
  if (mesh->nnx < 3 || mesh->nny < 3 || P.n_species < 1 || P.n_species > PIC_MAX_SPECIES ||
      !(P.dt > 0) || !(P.n_ref > 0) || !(P.T_ref_eV > 0) || P.pcg_maxit < 1 || !(P.pcg_tol > 0) ||
      mesh->n_objects < 0 || mesh->n_objects > PIC_MAX_OBJECTS) {
    set_error("pic_init: bad mesh size or parameters");
    return PIC_ERR_ARG;
  }
  if (P.precision != PIC_PREC_FP64 && P.precision != PIC_PREC_MIXED) {
    set_error("pic_init: unknown precision");
    return PIC_ERR_ARG;
  }
  if (mesh->delta != 0 && mesh->delta != 1) {
    set_error("pic_init: delta must be 0 (Cartesian) or 1 (axisymmetric)");
    return PIC_ERR_ARG;
  }
  if (mesh->delta == 1 && (!mesh->mass_rows || mesh->ymin != 0.0)) {
    set_error("pic_init: axisymmetric meshes need the per-row load matrices and the axis at ymin = 0");
    return PIC_ERR_ARG;
  }
  if ((int64_t)mesh->nnx * mesh->nny > (int64_t)1 << 30) {
    set_error("pic_init: mesh too large for int32 node ids");
    return PIC_ERR_ARG;
  }
  g = Ctx();
  g.P = P;
  g.axi = (mesh->delta == 1);
  g.solver = (P.solver == PIC_SOLVER_FCG_UNET) ? PIC_SOLVER_FCG_UNET : PIC_SOLVER_JPCG;
  if (g.P.sort_interval < 1) g.P.sort_interval = 1;
  MeshK &m = g.m;
  m.nnx = mesh->nnx;
  m.nny = mesh->nny;
  m.nex = m.nnx - 1;
  m.ney = m.nny - 1;
  m.xmin = mesh->xmin;
  m.xmax = mesh->xmax;
  m.ymin = mesh->ymin;
  m.ymax = mesh->ymax;
  m.hx = (m.xmax - m.xmin) / (m.nnx - 1);
  m.hy = (m.ymax - m.ymin) / (m.nny - 1);
  m.ney_magic = (uint32_t)((1ull << 32) / (unsigned)m.ney + 1ull);
  g.nn = (int64_t)m.nnx * m.nny;
  g.ne = (int64_t)m.nex * m.ney;
  const int64_t nn = g.nn, ne = g.ne;
  // reference scales, Input_2D.f90:362-392
  double T_ref = P.T_ref_eV * PIC_EVTOK;
  g.L_ref = std::sqrt(PIC_EPS0 * PIC_KB * T_ref / P.n_ref / PIC_QE / PIC_QE);
  g.t_ref = std::sqrt(PIC_EPS0 * PIC_ME / P.n_ref / PIC_QE / PIC_QE);
  g.v_ref = std::sqrt(PIC_KB * T_ref / PIC_ME);
  g.phi_ref = PIC_KB * T_ref / PIC_QE;

  int rc;
  PIC_CUDA(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
  PIC_CUDA(cudaStreamCreateWithFlags(&g.st2, cudaStreamNonBlocking));
  PIC_CUDA(cudaStreamCreateWithFlags(&g.st_copy, cudaStreamNonBlocking));
  for (auto &ev : g.step_ev) PIC_CUDA(cudaEventCreate(&ev));
  PIC_CUDA(cudaHostAlloc(&g.h_counters, 32 * sizeof(unsigned long long), cudaHostAllocMapped));
  PIC_CUDA(cudaHostGetDevicePointer((void **)&g.hd_counters, g.h_counters, 0));
  PIC_CUDA(cudaEventCreateWithFlags(&g.ev_copy_start, cudaEventDisableTiming));
  for (auto &ev : g.ev_field) PIC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  PIC_CUDA(cudaEventCreate(&g.ev0));
  PIC_CUDA(cudaEventCreate(&g.ev1));
  std::vector<double> xs(m.nnx), ys(m.nny);
  // node_x / node_y (the push) recompute these with the same expression
  for (int i = 0; i < m.nnx; ++i) xs[i] = m.xmin + m.hx * i;
  for (int j = 0; j < m.nny; ++j) ys[j] = m.ymin + m.hy * j;
  if ((rc = upload(&g.d_xs, xs.data(), xs.size()))) return rc;
  if ((rc = upload(&g.d_ys, ys.data(), ys.size()))) return rc;
  if ((rc = upload(&g.d_element_index, mesh->element_index, ne))) return rc;
  {
    // elements whose box meets an object's bounding box: only particles in
    // them can be inside an object (the mixed push tests objects there only)
    std::vector<uint8_t> near(ne, 0);
    const double hx = (mesh->xmax - mesh->xmin) / (mesh->nnx - 1), hy = (mesh->ymax - mesh->ymin) / (mesh->nny - 1);
    for (int k = 0; k < mesh->n_objects; ++k) {
      const pic_object &o = mesh->objects[k];
      double x0, x1, y0, y1;
      if (o.shape == PIC_SHAPE_BOX) {
        x0 = o.cx; x1 = o.a; y0 = o.cy; y1 = o.b;
      } else {
        const double hw = std::max(std::fabs(o.a), std::fabs(o.b)) * (1.0 + 1e-9);
        x0 = o.cx - hw; x1 = o.cx + hw; y0 = o.cy - hw; y1 = o.cy + hw;
      }
      const int i0 = std::max(0, (int)std::floor((x0 - mesh->xmin) / hx) - 1);
      const int i1 = std::min(mesh->nnx - 2, (int)std::floor((x1 - mesh->xmin) / hx) + 1);
      const int j0 = std::max(0, (int)std::floor((y0 - mesh->ymin) / hy) - 1);
      const int j1 = std::min(mesh->nny - 2, (int)std::floor((y1 - mesh->ymin) / hy) + 1);
      for (int i = i0; i <= i1; ++i)
        for (int j = j0; j <= j1; ++j) near[(size_t)i * (mesh->nny - 1) + j] = 1;
    }
    if ((rc = upload(&g.d_elem_near, near.data(), ne))) return rc;
  }
  if ((rc = upload(&g.d_node_index, mesh->node_index, nn))) return rc;
  if ((rc = upload(&g.d_node_type, mesh->node_type, nn))) return rc;
  if ((rc = upload(&g.d_phi_dir, mesh->phi_dirichlet, nn))) return rc;
  for (int w = 0; w < 2; ++w) {
    const int64_t i = (w == 0) ? 0 : m.nnx - 1;
    g.rf_ok[w] = true;
    for (int j = 0; j < m.nny; ++j) {
      const int64_t n = i * m.nny + j;
      if (mesh->node_type[n] > 0) {
        g.rf_ok[w] = false;
        continue;
      }
      const int reg = mesh->node_index[n];
      if (reg <= -2 && reg >= -(mesh->n_objects + 1) && mesh->objects[-reg - 2].conductor) continue;
      g.rf_line[w].push_back((int32_t)n);
      g.rf_base[w].push_back(mesh->phi_dirichlet[n]);
    }
  }
  if ((rc = upload(&g.d_cell_volume, mesh->cell_volume, nn))) return rc;
  const int nu = mesh->n_unknowns;
  std::vector<double> rhs_fix(nu, 0.0);
  if (mesh->rhs_fix) std::copy(mesh->rhs_fix, mesh->rhs_fix + nu, rhs_fix.begin());
  if ((rc = upload(&g.d_rhs_fix, rhs_fix.data(), rhs_fix.size()))) return rc;
  if ((rc = upload(&g.d_mass_q1, mesh->mass_q1, 16))) return rc;
  if ((rc = upload(&g.d_ife_mass, mesh->ife_mass, 16 * (size_t)mesh->n_interface))) return rc;
  if (g.axi && (rc = upload(&g.d_mass_rows, mesh->mass_rows, 16 * (size_t)m.ney))) return rc;
  ObjK ob;
  std::memset(&ob, 0, sizeof ob);
  ob.n = mesh->n_objects;
  for (int k = 0; k < ob.n; ++k) {
    ob.o[k] = mesh->objects[k];
    ob.ca[k] = std::cos(ob.o[k].angle);
    ob.sa[k] = std::sin(ob.o[k].angle);
    ob.half[k] = std::max(std::fabs(ob.o[k].a), std::fabs(ob.o[k].b)) * (1.0 + 1e-9);
  }
  PIC_CUDA(cudaMemcpyToSymbol(c_obj, &ob, sizeof ob));

  // validate every index table before it reaches a kernel
  {
    auto bad = [](const char *what) {
      set_error(std::string("pic_init: invalid ") + what);
      return PIC_ERR_ARG;
    };
    if (nu < 0 || nu > nn) return bad("n_unknowns");
    if (mesh->n_interface < 0 || (mesh->n_interface > 0 && !mesh->ife_mass)) return bad("interface data");
    for (int64_t e = 0; e < ne; ++e) {
      int v = mesh->element_index[e];
      if (v > mesh->n_interface || v == 0) return bad("element_index");
    }
    if (mesh->a_srow[0] != 1 || mesh->xt_srow[0] != 1) return bad("CSR row pointers");
    for (int u = 0; u < nu; ++u)
      if (mesh->a_srow[u + 1] < mesh->a_srow[u] || mesh->xt_srow[u + 1] < mesh->xt_srow[u])
        return bad("CSR row pointers");
    if (mesh->a_srow[nu] - 1 != mesh->nnz || mesh->xt_srow[nu] - 1 != mesh->nnz_xt) return bad("nnz");
    for (int64_t q = 0; q < mesh->nnz; ++q)
      if (mesh->a_jcol[q] < 1 || mesh->a_jcol[q] > nu) return bad("a_jcol");
    for (int64_t q = 0; q < mesh->nnz_xt; ++q)
      if (mesh->xt_jcol[q] < 1 || mesh->xt_jcol[q] > nn || mesh->node_type[mesh->xt_jcol[q] - 1] > 0)
        return bad("xt_jcol");
    if (mesh->patch_ptr[0] != 0) return bad("patch_ptr");
    for (int64_t n = 0; n < nn; ++n)
      if (mesh->patch_ptr[n + 1] < mesh->patch_ptr[n]) return bad("patch_ptr");
    for (int64_t q = 0; q < mesh->patch_ptr[nn]; ++q)
      if (mesh->patch_nodes[q] < 1 || mesh->patch_nodes[q] > nn) return bad("patch_nodes");
    for (int64_t n = 0; n < nn; ++n)
      if (!(mesh->cell_volume[n] > 0)) return bad("cell_volume");
  }
  // unknown id -> node map, sanity of the CSR
  std::vector<int32_t> u2n(nu, -1);
  for (int64_t n = 0; n < nn; ++n) {
    int t = mesh->node_type[n];
    if (t > 0) {
      if (t > nu) { set_error("pic_init: node_type out of range"); return PIC_ERR_ARG; }
      u2n[t - 1] = (int32_t)n;
    }
  }
  for (int u = 0; u < nu; ++u)
    if (u2n[u] < 0) { set_error("pic_init: unknown numbering has holes"); return PIC_ERR_ARG; }
  // A_xt rows in 0-based node columns
  {
    std::vector<int32_t> ptr(nu + 1), col;
    std::vector<double> val;
    for (int u = 0; u < nu; ++u) {
      ptr[u] = (int32_t)col.size();
      for (int64_t q = mesh->xt_srow[u] - 1; q < mesh->xt_srow[u + 1] - 1; ++q) {
        col.push_back(mesh->xt_jcol[q] - 1);
        val.push_back(mesh->xt_k[q]);
      }
    }
    ptr[nu] = (int32_t)col.size();
    if ((rc = upload(&g.d_xt_ptr, ptr.data(), ptr.size()))) return rc;
    if ((rc = upload(&g.d_xt_col, col.data(), col.size()))) return rc;
    if ((rc = upload(&g.d_xt_val, val.data(), val.size()))) return rc;
  }
  // split A into material stencils and explicit rows
  {
    const int nny = m.nny;
    auto row_entries = [&](int u, std::vector<std::pair<int64_t, double>> &out) {
      out.clear();
      for (int64_t q = mesh->a_srow[u] - 1; q < mesh->a_srow[u + 1] - 1; ++q)
        out.push_back({(int64_t)u2n[mesh->a_jcol[q] - 1], mesh->a_k[q]});
    };
    std::vector<std::pair<int64_t, double>> ent;
    g.n_mat = 0;
    // pass 1: stencils from rows whose four elements are one non-interface material
    for (int i = 1; i < m.nnx - 1 && g.n_mat < 16; ++i)
      for (int j = 1; j < nny - 1 && g.n_mat < 16; ++j) {
        int64_t n = (int64_t)i * nny + j;
        int u = mesh->node_type[n];
        if (u <= 0) continue;
        int e0 = mesh->element_index[(i - 1) * m.ney + (j - 1)];
        bool same = e0 < 0;
        for (int di = -1; di <= 0 && same; ++di)
          for (int dj = -1; dj <= 0 && same; ++dj)
            same = mesh->element_index[(i + di) * m.ney + (j + dj)] == e0;
        if (!same) continue;
        row_entries(u - 1, ent);
        if (ent.size() != 9) continue;
        double S[9];
        bool ok = true;
        for (int t = 0; t < 9 && ok; ++t) {
          int64_t want = n + (int64_t)(t / 3 - 1) * nny + (t % 3 - 1);
          ok = ent[t].first == want;
          S[t] = ent[t].second;
        }
        if (!ok) continue;
        bool known = false;
        for (int q = 0; q < g.n_mat && !known; ++q) known = std::memcmp(g.h_stencil[q], S, sizeof S) == 0;
        if (!known) std::memcpy(g.h_stencil[g.n_mat++], S, sizeof S);
      }
    std::vector<int32_t> kind(nn, -1), ex_cnt, ex_col;
    std::vector<double> ex_val, diag(nn, 1.0);
    for (int64_t n = 0; n < nn; ++n) {
      int u = mesh->node_type[n];
      if (u <= 0) continue;
      diag[n] = mesh->a_diag[u - 1];
      row_entries(u - 1, ent);
      int i = (int)(n / nny), j = (int)(n % nny);
      int mat = -1;
      if (i >= 1 && j >= 1 && i < m.nnx - 1 && j < nny - 1) {
        for (int q = 0; q < g.n_mat && mat < 0; ++q) {
          size_t pos = 0;
          bool ok = true;
          for (int t = 0; t < 9 && ok; ++t) {
            int64_t want = n + (int64_t)(t / 3 - 1) * nny + (t % 3 - 1);
            if (mesh->node_type[want] > 0) {
              ok = pos < ent.size() && ent[pos].first == want &&
                   std::memcmp(&ent[pos].second, &g.h_stencil[q][t], sizeof(double)) == 0;
              ++pos;
            }
          }
          if (ok && pos == ent.size()) mat = q;
        }
      }
      if (mat >= 0) {
        kind[n] = mat;
      } else {
        if (ent.size() > 9) {
          set_error("pic_init: stiffness row with more than 9 entries");
          return PIC_ERR_ARG;
        }
        kind[n] = g.n_mat + (int32_t)ex_cnt.size();
        ex_cnt.push_back((int32_t)ent.size());
        for (auto &pr : ent)
          if (pr.first < n - nny - 1 || pr.first > n + nny + 1) g.ex_local = false;
        for (size_t q = 0; q < 9; ++q) {
          ex_col.push_back(q < ent.size() ? (int32_t)ent[q].first : (int32_t)n);
          ex_val.push_back(q < ent.size() ? ent[q].second : 0.0);
        }
      }
    }
    PIC_CUDA(cudaMemcpyToSymbol(c_stencil, g.h_stencil, sizeof g.h_stencil));
    {
      float st32[16][9];
      for (int a = 0; a < 16; ++a)
        for (int c = 0; c < 9; ++c) st32[a][c] = (float)g.h_stencil[a][c];
      PIC_CUDA(cudaMemcpyToSymbol(c_stencil32, st32, sizeof st32));
      std::vector<float> ev32(ex_val.begin(), ex_val.end());
      if ((rc = upload(&g.d_ex_val32, ev32.data(), ev32.size()))) return rc;
    }
    if ((rc = upload(&g.d_row_kind, kind.data(), kind.size()))) return rc;
    if ((rc = upload(&g.d_ex_cnt, ex_cnt.data(), ex_cnt.size()))) return rc;
    if ((rc = upload(&g.d_ex_col, ex_col.data(), ex_col.size()))) return rc;
    if ((rc = upload(&g.d_ex_val, ex_val.data(), ex_val.size()))) return rc;
    if ((rc = upload(&g.d_diag, diag.data(), diag.size()))) return rc;
  }
  // PPR patches: regular 3x3 patches share one pseudo-inverse, others get their own rows
  {
    const int nny = m.nny;
    std::vector<int32_t> kind(nn, 2), ptr(nn + 1, 0), nodes;
    std::vector<double> rows, hs(nn, 1.0);
    {
      double h = std::max(m.hx, m.hy);
      std::vector<double> px, py;
      for (int a = -1; a <= 1; ++a)
        for (int b = -1; b <= 1; ++b) {
          px.push_back(a * m.hx / h);
          py.push_back(b * m.hy / h);
        }
      double R[45];
      if (!ppr_rows(px, py, R)) { set_error("pic_init: singular regular PPR patch"); return PIC_ERR_ARG; }
      for (int r = 0; r < 5; ++r)
        for (int q = 0; q < 9; ++q) g.h_ppr_reg[r][q] = R[r * 9 + q];
    }
    // patch layouts (relative node offsets in patch order) shared by at
    // least 1024 irregular nodes: one pseudo-inverse each, from the uniform
    // spacing, used where a node's own offsets match it to 1e-12
    std::map<std::vector<int32_t>, int64_t> layout_count;
    auto layout_of = [&](int64_t n, int b0, int cnt) {
      std::vector<int32_t> key(2 * cnt);
      const int i0 = (int)(n / nny), j0 = (int)(n % nny);
      for (int q = 0; q < cnt; ++q) {
        const int32_t mm = mesh->patch_nodes[b0 + q] - 1;
        key[2 * q] = mm / nny - i0;
        key[2 * q + 1] = mm % nny - j0;
      }
      return key;
    };
    for (int64_t n = 0; n < nn; ++n) {
      const int b0 = mesh->patch_ptr[n], cnt = mesh->patch_ptr[n + 1] - b0;
      if (cnt >= 6 && cnt != 9 && cnt <= kPprTplMax) ++layout_count[layout_of(n, b0, cnt)];
    }
    std::vector<std::pair<int64_t, std::vector<int32_t>>> common;
    for (auto &kv : layout_count)
      if (kv.second >= 1024) common.push_back({kv.second, kv.first});
    std::sort(common.begin(), common.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    if ((int)common.size() > kPprTpl) common.resize(kPprTpl);
    int tpl_cnt[kPprTpl] = {0}, tpl_off[kPprTpl][kPprTplMax] = {{0}};
    double tpl_R[kPprTpl][5][kPprTplMax] = {{{0}}};
    std::vector<std::vector<double>> tpl_px(common.size()), tpl_py(common.size());
    int ntpl = 0;
    for (auto &cl : common) {
      const std::vector<int32_t> &key = cl.second;
      const int cnt = (int)key.size() / 2;
      double h = 0.0;
      for (int q = 0; q < cnt; ++q) h = std::max(h, std::max(std::fabs(key[2 * q] * m.hx), std::fabs(key[2 * q + 1] * m.hy)));
      std::vector<double> px(cnt), py(cnt), R(5 * cnt);
      for (int q = 0; q < cnt; ++q) {
        px[q] = key[2 * q] * m.hx / h;
        py[q] = key[2 * q + 1] * m.hy / h;
      }
      if (!ppr_rows(px, py, R.data())) continue;
      tpl_cnt[ntpl] = cnt;
      for (int q = 0; q < cnt; ++q) {
        tpl_off[ntpl][q] = key[2 * q] * nny + key[2 * q + 1];
        for (int r = 0; r < 5; ++r) tpl_R[ntpl][r][q] = R[(size_t)r * cnt + q];
      }
      tpl_px[ntpl] = px;
      tpl_py[ntpl] = py;
      layout_count[key] = -1 - ntpl;  // marks the layout as template ntpl
      ++ntpl;
    }
    for (int64_t n = 0; n < nn; ++n) {
      ptr[n] = (int32_t)nodes.size();
      int b0 = mesh->patch_ptr[n], cnt = mesh->patch_ptr[n + 1] - b0;
      int i = (int)(n / nny), j = (int)(n % nny);
      double xi = xs[i], yi = ys[j];
      double h = 0.0;
      for (int q = 0; q < cnt; ++q) {
        int32_t mm = mesh->patch_nodes[b0 + q] - 1;
        double dx = std::fabs(xs[mm / nny] - xi), dy = std::fabs(ys[mm % nny] - yi);
        h = std::max(h, std::max(dx, dy));
      }
      hs[n] = (h > 0) ? h : 1.0;
      if (cnt < 6) continue;
      bool regular = (cnt == 9) && i >= 1 && j >= 1 && i < m.nnx - 1 && j < nny - 1;
      for (int t = 0; t < 9 && regular; ++t)
        regular = (mesh->patch_nodes[b0 + t] - 1) == n + (int64_t)(t / 3 - 1) * nny + (t % 3 - 1);
      if (regular) {
        kind[n] = 0;
        continue;
      }
      std::vector<double> px(cnt), py(cnt);
      for (int q = 0; q < cnt; ++q) {
        int32_t mm = mesh->patch_nodes[b0 + q] - 1;
        px[q] = (xs[mm / nny] - xi) / h;
        py[q] = (ys[mm % nny] - yi) / h;
      }
      if (ntpl > 0 && cnt <= kPprTplMax && cnt != 9) {
        auto it = layout_count.find(layout_of(n, b0, cnt));
        if (it != layout_count.end() && it->second < 0) {
          const int t = (int)(-1 - it->second);
          bool same = true;
          for (int q = 0; q < cnt && same; ++q)
            same = std::fabs(px[q] - tpl_px[t][q]) <= 1e-12 && std::fabs(py[q] - tpl_py[t][q]) <= 1e-12;
          if (same) {
            kind[n] = 3 + t;
            continue;
          }
        }
      }
      std::vector<double> R(5 * cnt);
      if (!ppr_rows(px, py, R.data())) continue;  // singular patch: no recovery at this node
      kind[n] = 1;
      ptr[n] = (int32_t)nodes.size();
      for (int q = 0; q < cnt; ++q) nodes.push_back(mesh->patch_nodes[b0 + q] - 1);
      rows.insert(rows.end(), R.begin(), R.end());
    }
    ptr[nn] = (int32_t)nodes.size();
    // kind 1 rows are stored at 5*ptr[n]; ptr for kinds 0/2 is unused
    PIC_CUDA(cudaMemcpyToSymbol(c_ppr_reg, g.h_ppr_reg, sizeof g.h_ppr_reg));
    PIC_CUDA(cudaMemcpyToSymbol(c_ppr_tpl_cnt, tpl_cnt, sizeof tpl_cnt));
    PIC_CUDA(cudaMemcpyToSymbol(c_ppr_tpl_off, tpl_off, sizeof tpl_off));
    PIC_CUDA(cudaMemcpyToSymbol(c_ppr_tpl_R, tpl_R, sizeof tpl_R));
    if ((rc = upload(&g.d_ppr_kind, kind.data(), kind.size()))) return rc;
    // make ptr monotone for kind-1 lookups: ptr[n+1] must be the end of node n's patch
    std::vector<int32_t> ptr2(nn + 1, 0);
    {
      int32_t acc = 0;
      for (int64_t n = 0; n < nn; ++n) {
        ptr2[n] = acc;
        if (kind[n] == 1) {
          int b0 = mesh->patch_ptr[n], cnt = mesh->patch_ptr[n + 1] - b0;
          acc += cnt;
        }
      }
      ptr2[nn] = acc;
    }
    if ((rc = upload(&g.d_ppr_ptr, ptr2.data(), ptr2.size()))) return rc;
    if ((rc = upload(&g.d_ppr_nodes, nodes.data(), nodes.size()))) return rc;
    if ((rc = upload(&g.d_ppr_rows, rows.data(), rows.size()))) return rc;
    if ((rc = upload(&g.d_ppr_h, hs.data(), hs.size()))) return rc;
  }
  // fields and solver vectors
  if ((rc = dalloc(&g.d_phi, nn))) return rc;
  if ((rc = dalloc(&g.d_rho, nn))) return rc;
  if ((rc = dalloc(&g.d_efx, nn))) return rc;
  if ((rc = dalloc(&g.d_efy, nn))) return rc;
  if ((rc = dalloc(&g.d_coef, 5 * nn))) return rc;
  PIC_CUDA(cudaMemset(g.d_efx, 0, nn * sizeof(double)));
  PIC_CUDA(cudaMemset(g.d_efy, 0, nn * sizeof(double)));
  PIC_CUDA(cudaMemset(g.d_coef, 0, 5 * nn * sizeof(double)));
  g.mixed = (P.precision == PIC_PREC_MIXED);
  if (g.mixed) {
    if ((rc = dalloc(&g.d_coef32, 8 * nn))) return rc;
    PIC_CUDA(cudaMemset(g.d_coef32, 0, 8 * nn * sizeof(float)));
  }
  // every context (a species can hold FP64 particles in a mixed one)
  if ((rc = dalloc(&g.d_efxy, nn))) return rc;
  PIC_CUDA(cudaMemset(g.d_efxy, 0, nn * sizeof(double2)));
  PIC_CUDA(cudaMemset(g.d_rho, 0, nn * sizeof(double)));
  PIC_CUDA(cudaMemcpy(g.d_phi, mesh->phi_dirichlet, nn * sizeof(double), cudaMemcpyHostToDevice));
  for (double **v : {&g.d_b, &g.d_x, &g.d_r, &g.d_w, &g.d_p[0], &g.d_p[1], &g.d_q}) {
    if ((rc = dalloc(v, nn))) return rc;
    PIC_CUDA(cudaMemset(*v, 0, nn * sizeof(double)));
  }
  g.red_blocks = (int)((nn + PIC_RED_CHUNK - 1) / PIC_RED_CHUNK);
  if ((rc = dalloc(&g.d_part, 3 * (size_t)g.red_blocks))) return rc;
  if ((rc = dalloc(&g.d_pcg, 1))) return rc;
  PIC_CUDA(cudaMemset(g.d_pcg, 0, sizeof(PcgState)));
  if ((rc = dalloc(&g.d_bar, 4))) return rc;
  PIC_CUDA(cudaMemset(g.d_bar, 0, 4 * sizeof(unsigned int)));
  if ((rc = dalloc(&g.d_z, nn))) return rc;
  PIC_CUDA(cudaMemset(g.d_z, 0, nn * sizeof(double)));
  if ((rc = dalloc(&g.d_dot, 2))) return rc;
  if ((rc = dalloc(&g.d_dot_ticket, 1))) return rc;
  PIC_CUDA(cudaMemset(g.d_dot_ticket, 0, sizeof(unsigned int)));
  if ((rc = dalloc(&g.d_fcg, 1))) return rc;
  PIC_CUDA(cudaMemset(g.d_fcg, 0, sizeof(FcgState)));
  {
    // persistent PCG when the device supports cooperative launch and every
    // CTA of the grid can be resident at once
    int dev = 0, coop = 0, nsm = 0, per_sm = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    PIC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    PIC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_persist, kWide, 0));
    const char *env = getenv("PIC_PCG_PERSISTENT");
    bool want = !(env && env[0] == '0');
    g.coop_grid = (want && coop && per_sm > 0) ? std::min(g.red_blocks, per_sm * nsm) : 0;
    int per_sm_f = 0;
    int per_sm_f32 = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, k_fcg_persist<double>, kWide, 0));
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f32, k_fcg_persist<float>, kWide, 0));
    per_sm_f = std::min(per_sm_f, per_sm_f32);
    const char *envf = getenv("PIC_FCG_PERSISTENT");
    const bool want_f = !(envf && envf[0] == '0');
    g.fcg_coop_grid = (want_f && coop && per_sm_f > 0) ? std::min(g.red_blocks, per_sm_f * nsm) : 0;
    // shared-memory-resident variant: every CTA owns at most kSmemChunks
    // chunks and its window of w and p fits next to them
    g.smem_grid = 0;
    const char *env2 = getenv("PIC_PCG_SMEM");
    bool want_smem = want && !(env2 && env2[0] == '0');
    const int H = m.nny + 1;
    const size_t bytes = (size_t)(2 * (kSmemChunks * kWide + 2 * H) + 5 * kSmemChunks * kWide) * sizeof(double);
    int max_smem = 0;
    PIC_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (want_smem && coop && g.ex_local && bytes + 2048 <= (size_t)max_smem) {
      PIC_CUDA(cudaFuncSetAttribute(k_pcg_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
      int per_sm2 = 0;
      PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_pcg_smem, kWide, bytes));
      int G = std::min(g.red_blocks, per_sm2 * nsm);
      if (per_sm2 > 0 && (int64_t)G * kSmemChunks >= g.red_blocks) {
        g.smem_grid = G;
        g.smem_bytes = bytes;
      }
    }
    // failure-path test hooks: a short wait limit and an arrival that never comes
    const char *lim = getenv("PIC_PCG_SPIN_LIMIT");
    g.pcg_spin_limit = lim ? std::max(1ll, atoll(lim)) : (1ll << 22);
    const char *extra = getenv("PIC_PCG_BARRIER_EXTRA");
    g.pcg_bar_extra = extra ? (unsigned int)std::max(0, atoi(extra)) : 0u;
  }
  {
    const char *ff = getenv("PIC_FCG_FUSED");  // 0: the persistent FCG's set-up and judge by separate kernels
    g.fcg_fused = (ff && atoi(ff) == 0) ? 0 : 1;
    const char *fg = getenv("PIC_FCG_GRAPHS");  // 0: enqueue FCG iterations kernel by kernel
    g.fcg_graphs = (fg && atoi(fg) == 0) ? 0 : 1;
    const char *fi = getenv("PIC_FCG_INNER");  // "fp32": FP32 inner iterations in mixed precision
    g.fcg_inner32 = (fi && std::strcmp(fi, "fp32") == 0) ? 1 : 0;
    // mixed-precision push: particle tiles staged through shared memory
    // with S-stage cp.async (2..4; 4 by default: 2.56 ms against 2.81 ms per
    // step at 101M particles), or 0 for one particle per thread loaded
    // directly
    const char *mf = getenv("PIC_MCC_FULL");  // 1: MCC selection by the full key histogram
    g.mcc_full = (mf && atoi(mf) == 1) ? 1 : 0;
    const char *mps = getenv("PIC_MCC_PUSH_SELECT");  // 0: the MCC pass reads the particles itself
    g.mcc_push_select = mps ? atoi(mps) != 0 : true;
    const char *mb2 = getenv("PIC_MCC_BOUND_SCALE");  // test hook (see mcc_bound_scale)
    g.mcc_bound_scale = mb2 ? std::max(1e-6, atof(mb2)) : 1.0;
    const char *ps = getenv("PIC_PUSH_STAGES");
    g.push_stages = ps ? atoi(ps) : g.push_stages;
    if (g.push_stages != 0 && (g.push_stages < 2 || g.push_stages > 4)) g.push_stages = 0;
    int dev = 0, nsm = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    PIC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    g.push_grid = 0;
    if (g.push_stages) {
      // resident CTAs per SM the 4-stage kernel is compiled for: 5 (48
      // registers) measured 2.42 ms/step against 2.56 with 4 (56 registers)
      // and 2.43 with 6 (40 registers, small spills)
      const char *mb = getenv("PIC_PUSH_MINB");
      g.push_minb = mb ? atoi(mb) : g.push_minb;
      if (g.axi) g.push_stages = 4;  // the r-z push has the 4-stage, 5-CTA form only
      const void *fn = g.axi                ? (const void *)k_push_mixed_tiled<4, 5, true>
                       : g.push_stages == 2 ? (const void *)k_push_mixed_tiled<2>
                       : g.push_stages == 3 ? (const void *)k_push_mixed_tiled<3>
                       : g.push_minb == 5   ? (const void *)k_push_mixed_tiled<4, 5>
                       : g.push_minb == 6   ? (const void *)k_push_mixed_tiled<4, 6>
                                            : (const void *)k_push_mixed_tiled<4>;
      // PIC_PUSH_BULK=1 (default): the 4-stage, 5-CTA form with tiles
      // bulk-copied by one thread and completing on mbarriers
      const char *pb = getenv("PIC_PUSH_BULK");
      g.push_bulk = (pb ? atoi(pb) == 1 : g.push_bulk_default) && g.push_stages == 4 && (g.axi || g.push_minb == 5);
      if (g.push_bulk)
        fn = g.axi ? (const void *)k_push_mixed_bulk<4, 5, true> : (const void *)k_push_mixed_bulk<4, 5, false>;
      int per_sm = 0;
      PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, fn, kPushTile, (size_t)g.push_stages * sizeof(PushTile) + (g.push_bulk ? 4 * sizeof(uint64_t) : 0)));
      g.push_grid = per_sm * nsm;
      if (g.push_grid <= 0) g.push_stages = 0;
    }
    // FP64 push: particle tiles (9 KB each, 3 stages = 27 KB per CTA) staged
    // through shared memory when PIC_PUSH64_TILED is 1; otherwise one
    // particle per thread loaded directly (same bits either way)
    // (2: the tiles are bulk-copied by one thread and complete on mbarriers)
    // test hooks of the bulk-staged pushes' bounded wait: polls of a tile's
    // mbarrier before giving up, and no copies issued at all (every wait then
    // runs out and the step reports the failure)
    const char *wl = getenv("PIC_PUSH_WAIT_LIMIT");
    if (wl && atoll(wl) > 0) g.push_wait_limit = atoll(wl);
    const char *sc = getenv("PIC_PUSH_SKIP_COPIES");
    g.push_skip_copies = sc && atoi(sc) == 1 ? 1 : 0;
    const char *p64 = getenv("PIC_PUSH64_TILED");
    const int mode64 = p64 ? atoi(p64) : g.push64_default;
    g.push64_grid = 0;
    g.push64_bulk = mode64 == 2;
    if (mode64 == 1 || mode64 == 2) {
      const char *m64 = getenv("PIC_PUSH64_MINB");  // 5: the Cartesian bulk push built for 5 CTAs per SM
      g.push64_minb = (m64 && atoi(m64) == 5 && !g.axi) ? 5 : 4;
      const void *fn = g.push64_bulk ? (g.axi ? (const void *)k_push_bulk<3, true>
                                              : g.push64_minb == 5 ? (const void *)k_push_bulk<3, false, 5>
                                                                   : (const void *)k_push_bulk<3, false>)
                                     : (g.axi ? (const void *)k_push_tiled<3, true> : (const void *)k_push_tiled<3, false>);
      const size_t smem = 3 * sizeof(PushTile64) + (g.push64_bulk ? 3 * sizeof(uint64_t) : 0);
      int per_sm = 0;
      PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPushTile, smem));
      g.push64_grid = per_sm * nsm;
    }
  }
  if ((rc = dalloc(&g.d_counters, 32))) return rc;
  PIC_CUDA(cudaMemset(g.d_counters, 0, 32 * sizeof(unsigned long long)));
  // sort scratch sized for the largest species
  if ((rc = dalloc(&g.d_cell_count, ne + 1))) return rc;
  if ((rc = dalloc(&g.d_cell_start, ne + 1))) return rc;
  if ((rc = dalloc(&g.d_cell_fill, ne + 1))) return rc;
  if ((rc = dalloc(&g.d_scan_blk, 4100))) return rc;
  int64_t maxcap = 1;
  g.ns = P.n_species;
  for (int s = 0; s < g.ns; ++s) {
    Species &sp = g.sp[s];
    const pic_species_desc &d = P.species[s];
    if (!(d.mass > 0) || d.capacity < 0 || d.capacity > ((int64_t)1 << 31) - 1) {
      set_error("pic_init: bad species description");
      free_all();
      return PIC_ERR_ARG;
    }
    sp.charge = d.charge;
    sp.mass = d.mass;
    sp.weight = d.weight;
    sp.qm = d.charge / (d.mass / PIC_ME);
    sp.capacity = d.capacity;
    sp.f32 = (P.precision == PIC_PREC_MIXED);
    maxcap = std::max(maxcap, d.capacity);
    // whole 256-particle tiles, so that a push tile copy never reads past
    // the allocation
    size_t c = (size_t)(std::max<int64_t>(d.capacity, 1) + kPushTile - 1) / kPushTile * kPushTile;
    for (double **v : {&sp.x, &sp.y, &sp.vx, &sp.vy, &sp.vz, &sp.x2, &sp.y2, &sp.vx2, &sp.vy2, &sp.vz2})
      if ((rc = dalloc(v, c))) return rc;
    if ((rc = dalloc(&sp.loc, c))) return rc;
    if ((rc = dalloc(&sp.loc2, c))) return rc;
    if ((rc = dalloc(&sp.id, c))) return rc;
    if ((rc = dalloc(&sp.id2, c))) return rc;
    if ((rc = dalloc(&sp.q_acc, nn))) return rc;
    if ((rc = dalloc(&sp.e_acc, nn))) return rc;
    if ((rc = dalloc(&sp.rho_s, nn))) return rc;
    if ((rc = dalloc(&sp.ek_s, nn))) return rc;
    if ((rc = dalloc(&sp.ek_tot, nn))) return rc;
    PIC_CUDA(cudaMemset(sp.q_acc, 0, nn * sizeof(unsigned long long)));
    PIC_CUDA(cudaMemset(sp.e_acc, 0, nn * sizeof(unsigned long long)));
    PIC_CUDA(cudaMemset(sp.rho_s, 0, nn * sizeof(double)));
    PIC_CUDA(cudaMemset(sp.ek_s, 0, nn * sizeof(double)));
    PIC_CUDA(cudaMemset(sp.ek_tot, 0, nn * sizeof(double)));
  }
  if ((rc = dalloc(&g.d_perm, maxcap))) return rc;
  if ((rc = dalloc(&g.d_perm2, maxcap))) return rc;
  if ((rc = dalloc(&g.d_sort_id, maxcap))) return rc;
  PIC_CUDA(cudaDeviceSynchronize());
  g.inited = true;
  return PIC_OK;
}

int pic_upload_particles(int32_t species, int64_t n, const double *x, const double *y,
                         const double *vx, const double *vy, const double *vz, const int32_t *loc,
                         const uint32_t *id) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  Species &s = g.sp[species];
  if (n < 0 || (n > 0 && (!x || !y || !vx || !vy || !vz))) {
    set_error("pic_upload_particles: bad arguments");
    return PIC_ERR_ARG;
  }
  if (n > s.capacity) {
    set_error("pic_upload_particles: more particles than the species capacity");
    return PIC_ERR_CAPACITY;
  }
  size_t b = (size_t)n * sizeof(double);
  PIC_CUDA(cudaMemcpyAsync(s.x, x, b, cudaMemcpyHostToDevice, g.st));
  PIC_CUDA(cudaMemcpyAsync(s.y, y, b, cudaMemcpyHostToDevice, g.st));
  PIC_CUDA(cudaMemcpyAsync(s.vx, vx, b, cudaMemcpyHostToDevice, g.st));
  PIC_CUDA(cudaMemcpyAsync(s.vy, vy, b, cudaMemcpyHostToDevice, g.st));
  PIC_CUDA(cudaMemcpyAsync(s.vz, vz, b, cudaMemcpyHostToDevice, g.st));
  std::vector<uint32_t> ids;
  if (!id) {
    ids.resize(n);
    for (int64_t k = 0; k < n; ++k) ids[k] = (uint32_t)k;
    id = ids.data();
  }
  uint32_t mx = 0;
  for (int64_t k = 0; k < n; ++k) mx = std::max(mx, id[k]);
  PIC_CUDA(cudaMemcpyAsync(s.id, id, (size_t)n * 4, cudaMemcpyHostToDevice, g.st));
  s.n_slots = n;
  s.n_live = n;
  s.next_id = n ? mx + 1 : 0;
  if (loc) {
    for (int64_t k = 0; k < n; ++k)
      if (loc[k] < -1 || loc[k] >= g.ne) {
        s.n_slots = s.n_live = 0;
        set_error("pic_upload_particles: element index out of range");
        return PIC_ERR_ARG;
      }
    PIC_CUDA(cudaMemcpyAsync(s.loc, loc, (size_t)n * 4, cudaMemcpyHostToDevice, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
  } else {
    if (int rc_ = zero_async(s.loc, (size_t)n * 4, g.st)) return rc_;
    if ((rc = zero_counter(1))) return rc;
    if ((rc = launch_locate(s, 0, n))) return rc;
    unsigned long long bad = 0;
    if ((rc = read_counter(1, &bad))) return rc;
    if (bad) {
      set_error("pic_upload_particles: particle outside the mesh");
      return PIC_ERR_DOMAIN;
    }
  }
  if (s.f32 && (rc = to_mixed(s))) return rc;
  return PIC_OK;
}

int pic_particle_count(int32_t species, int64_t *n) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  if (n) *n = g.sp[species].n_live;
  return PIC_OK;
}

int pic_get_next_id(int32_t species, uint32_t *next_id) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  if (!next_id) {
    set_error("pic_get_next_id: null output");
    return PIC_ERR_ARG;
  }
  *next_id = g.sp[species].next_id;
  return PIC_OK;
}

int pic_set_next_id(int32_t species, uint32_t next_id) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  if (next_id < g.sp[species].next_id) {
    set_error("pic_set_next_id: below the largest id in use + 1 (ids would repeat)");
    return PIC_ERR_ARG;
  }
  g.sp[species].next_id = next_id;
  return PIC_OK;
}

int pic_download_particles(int32_t species, int64_t capacity, double *x, double *y, double *vx,
                           double *vy, double *vz, int32_t *loc, uint32_t *id, int64_t *n_out) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  Species &s = g.sp[species];
  // compact on the host side: copy all slots, keep live ones in order
  int64_t ns = s.n_slots;
  std::vector<int32_t> hl(ns);
  PIC_CUDA(cudaMemcpyAsync(hl.data(), s.loc, ns * 4, cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  int64_t live = 0;
  for (int64_t k = 0; k < ns; ++k) live += hl[k] >= 0;
  if (n_out) *n_out = live;
  if (live > capacity) {
    set_error("pic_download_particles: output capacity too small");
    return PIC_ERR_CAPACITY;
  }
  auto pull = [&](const void *src, void *dst, size_t esz) -> int {
    if (!dst) return PIC_OK;
    std::vector<char> tmp(ns * esz);
    PIC_CUDA(cudaMemcpy(tmp.data(), src, ns * esz, cudaMemcpyDeviceToHost));
    int64_t o = 0;
    for (int64_t k = 0; k < ns; ++k)
      if (hl[k] >= 0) std::memcpy((char *)dst + (o++) * esz, tmp.data() + k * esz, esz);
    return PIC_OK;
  };
  const double *sx = s.x, *sy = s.y, *svx = s.vx, *svy = s.vy, *svz = s.vz;
  if (s.f32) {  // absolute FP64 values into the staging set
    if ((rc = from_mixed(s))) return rc;
    PIC_CUDA(cudaStreamSynchronize(g.st));
    sx = s.x2;
    sy = s.y2;
    svx = s.vx2;
    svy = s.vy2;
    svz = s.vz2;
  }
  if ((rc = pull(sx, x, 8)) || (rc = pull(sy, y, 8)) || (rc = pull(svx, vx, 8)) ||
      (rc = pull(svy, vy, 8)) || (rc = pull(svz, vz, 8)) || (rc = pull(s.loc, loc, 4)) ||
      (rc = pull(s.id, id, 4)))
    return rc;
  return PIC_OK;
}

int pic_particle_device_ptrs(int32_t species, void **ptrs7, int64_t *n_slots) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  Species &s = g.sp[species];
  if (s.f32) {
    // The FP32 element-offset layout is not the documented double* one: hand
    // it to no zero-copy caller (a deposit or diagnostic fed from it would
    // read FP32 offsets as FP64 positions without any error).
    set_error("pic_particle_device_ptrs: the particles are stored in the mixed-precision layout "
              "(FP32 element offsets and velocities), not as FP64 positions; use "
              "pic_download_particles");
    return PIC_ERR_STATE;
  }
  if (ptrs7) {
    ptrs7[0] = s.x; ptrs7[1] = s.y; ptrs7[2] = s.vx; ptrs7[3] = s.vy; ptrs7[4] = s.vz;
    ptrs7[5] = s.loc; ptrs7[6] = s.id;
  }
  if (n_slots) *n_slots = s.n_slots;
  return PIC_OK;
}

int pic_particle_positioning(int32_t species) {
  int rc;
  if ((rc = check_init())) return rc;
  int s0 = species < 0 ? 0 : species, s1 = species < 0 ? g.ns : species + 1;
  if (species >= 0 && (rc = check_species(species))) return rc;
  if ((rc = zero_counter(1))) return rc;
  for (int s = s0; s < s1; ++s)  // mixed precision: the element is part of the position
    if (!g.sp[s].f32 && (rc = launch_locate(g.sp[s], 0, g.sp[s].n_slots))) return rc;
  unsigned long long bad = 0;
  if ((rc = read_counter(1, &bad))) return rc;
  if (bad) {
    set_error("pic_particle_positioning: particle outside the mesh");
    return PIC_ERR_DOMAIN;
  }
  return PIC_OK;
}

// the bulk-staged FP64 push counts the tiles whose bounded wait ran out
static int check_push_fail(const char *who) {
  unsigned long long fail = 0;
  int rc = read_counter(2, &fail);
  if (rc) return rc;
  if (fail) {
    zero_counter(2);
    set_error(std::string(who) + ": a push tile copy did not complete within its bounded wait");
    return PIC_ERR_CUDA;
  }
  return PIC_OK;
}

static int count_live(int sidx) {
  Species &s = g.sp[sidx];
  unsigned long long lost = 0;
  int rc = read_counter(8 + sidx, &lost);
  if (rc) return rc;
  s.n_live -= (int64_t)lost;
  return zero_counter(8 + sidx);
}

int pic_move_all(int32_t species, int32_t push_flag) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  (void)push_flag;
  if ((rc = zero_counter(8 + species))) return rc;
  if ((rc = run_push(species, true, false, false))) return rc;
  if ((rc = check_push_fail("pic_move_all"))) return rc;
  return count_live(species);
}

int pic_get_par_chg(int32_t delta, double *rho_out) {
  int rc;
  if ((rc = check_init())) return rc;
  if ((rc = fields_fence(0xFu))) return rc;
  if (delta != (g.axi ? 1 : 0)) {
    set_error("pic_get_par_chg: delta differs from the mesh's");
    return PIC_ERR_ARG;
  }
  if ((rc = zero_deposit(true))) return rc;
  if ((rc = zero_counter(1))) return rc;
  for (int s = 0; s < g.ns; ++s) {
    if ((rc = zero_counter(8 + s))) return rc;
    if ((rc = run_push(s, false, true, true))) return rc;
    if ((rc = count_live(s))) return rc;
  }
  if ((rc = run_rho(true))) return rc;
  unsigned long long bad = 0;
  if ((rc = read_counter(1, &bad))) return rc;
  if (bad) {
    set_error("pic_get_par_chg: particle outside the mesh");
    return PIC_ERR_DOMAIN;
  }
  if (rho_out) {
    PIC_CUDA(cudaMemcpyAsync(rho_out, g.d_rho, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st));
    PIC_CUDA(cudaStreamSynchronize(g.st));
  }
  return PIC_OK;
}

int pic_ife_solve(double *phi_inout, double time, pic_solve_stats *stats) {
  int rc;
  if ((rc = check_init())) return rc;
  if ((rc = fields_fence(0xFu))) return rc;
  if (phi_inout)
    PIC_CUDA(cudaMemcpyAsync(g.d_phi, phi_inout, g.nn * sizeof(double), cudaMemcpyHostToDevice, g.st));
  PIC_CUDA(cudaEventRecord(g.ev0, g.st));
  if ((rc = rf_apply(time))) return rc;
  if ((rc = run_rhs())) return rc;
  int src = run_solve(stats);
  PIC_CUDA(cudaEventRecord(g.ev1, g.st));
  if (phi_inout)
    PIC_CUDA(cudaMemcpyAsync(phi_inout, g.d_phi, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, g.ev0, g.ev1);
    stats->ms = ms;
  }
  return src;
}

int pic_set_wall_rf(int32_t wall, double amplitude, double frequency_hz, double phase) {
  int rc;
  if ((rc = check_init())) return rc;
  if (wall < 0 || wall > 1 || !std::isfinite(amplitude) || !std::isfinite(frequency_hz) || !std::isfinite(phase)) {
    set_error("pic_set_wall_rf: wall must be 0 (x = xmin) or 1 (x = xmax), values finite");
    return PIC_ERR_ARG;
  }
  if (amplitude != 0.0 && !g.rf_ok[wall]) {
    set_error("pic_set_wall_rf: the wall is not a Dirichlet wall");
    return PIC_ERR_ARG;
  }
  if ((rc = fields_fence(0x2u))) return rc;  // writes phi
  // the previous wall back to its static values
  if (g.rf_wall >= 0 && g.rf_count > 0) {
    k_rf_set<<<(g.rf_count + 127) / 128, 128, 0, g.st>>>(g.d_rf_nodes, g.d_rf_base, g.rf_count, 0.0, g.d_phi_dir,
                                                        g.d_phi);
    PIC_LAUNCHED();
  }
  PIC_CUDA(cudaStreamSynchronize(g.st));
  if (g.d_rf_nodes) cudaFree(g.d_rf_nodes);
  if (g.d_rf_base) cudaFree(g.d_rf_base);
  g.d_rf_nodes = nullptr;
  g.d_rf_base = nullptr;
  g.rf_wall = -1;
  g.rf_count = 0;
  if (amplitude == 0.0) return PIC_OK;
  const size_t cnt = g.rf_line[wall].size();
  if ((rc = upload(&g.d_rf_nodes, g.rf_line[wall].data(), cnt))) return rc;
  if ((rc = upload(&g.d_rf_base, g.rf_base[wall].data(), cnt))) return rc;
  g.rf_wall = wall;
  g.rf_count = (int)cnt;
  g.rf_amp = amplitude;
  g.rf_omega = (2.0 * M_PI * frequency_hz) * g.t_ref;
  g.rf_phase = phase;
  return PIC_OK;
}

int pic_get_efield_ppr(double *efx_out, double *efy_out) {
  int rc;
  if ((rc = check_init())) return rc;
  if ((rc = fields_fence(0xFu))) return rc;
  if ((rc = run_ppr())) return rc;
  if (efx_out)
    PIC_CUDA(cudaMemcpyAsync(efx_out, g.d_efx, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  if (efy_out)
    PIC_CUDA(cudaMemcpyAsync(efy_out, g.d_efy, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  return PIC_OK;
}

int pic_sort_particles(int32_t species) {
  int rc;
  if ((rc = check_init()) || (rc = check_species(species))) return rc;
  return sort_species(species);
}

int pic_step(uint64_t step, pic_step_stats *stats) {
  int rc;
  if ((rc = check_init())) return rc;
  cudaEvent_t *e = g.step_ev;  // created once, at pic_init
  PIC_CUDA(cudaEventRecord(e[0], g.st));
  // 1. fused push + locate + deposit (MoveAll, then GetParChg_2D).  The
  // per-node energy (Ek_tot) is a diagnostic the reference only writes at its
  // output cadence: it is deposited on steps that are multiples of
  // diag_interval (every step when diag_interval <= 1).
  const bool diag = g.P.diag_interval <= 1 || (step % (uint64_t)g.P.diag_interval) == 0;
  if ((rc = zero_deposit(diag))) return rc;
  if ((rc = zero_counter(1))) return rc;
  int64_t before[PIC_MAX_SPECIES];
  int64_t pushed = 0;
  for (int s = 0; s < g.ns; ++s) {
    before[s] = g.sp[s].n_live;
    pushed += before[s];
    if ((rc = zero_counter(8 + s))) return rc;
  }
  // the MCC selection of this step is built by the push itself
  if (g.mcc_ready && g.mcc_push_select && (rc = mcc_prepare(step))) return rc;
  PIC_CUDA(cudaEventRecord(e[6], g.st));
  g.sel_push = g.sel_step == step;
  for (int s = 0; s < g.ns; ++s)
    if ((rc = run_push(s, true, true, diag))) {
      g.sel_push = false;
      return rc;
    }
  g.sel_push = false;
  PIC_CUDA(cudaEventRecord(e[7], g.st));
  // the fields' writers (deposit, solve, field recovery) follow the copies
  // of the previous step's fields, which ran alongside the push
  if ((rc = fields_fence(0xFu))) return rc;
  if ((rc = run_rho(diag))) return rc;
  PIC_CUDA(cudaEventRecord(e[1], g.st));
  // 2. Poisson (IFE_Solve_2D)
  pic_solve_stats ss;
  std::memset(&ss, 0, sizeof ss);
  if ((rc = rf_apply((double)step * g.P.dt))) return rc;  // xt = it*dt (Main_IFE_Test_2.f90:279)
  if ((rc = run_rhs())) return rc;
  int solve_rc = run_solve(&ss);
  PIC_CUDA(cudaEventRecord(e[2], g.st));
  // 3. PPR field recovery, on the second stream alongside the MCC: the PPR
  // reads phi and writes the fields, the MCC reads and writes particles only
  PIC_CUDA(cudaEventRecord(e[3], g.st));
  PIC_CUDA(cudaStreamWaitEvent(g.st2, e[3], 0));
  PIC_CUDA(cudaEventRecord(e[8], g.st2));
  if ((rc = run_ppr(g.st2))) return rc;
  PIC_CUDA(cudaEventRecord(e[9], g.st2));
  {  // the particles each species lost in the push, one read for all
    unsigned long long lost[PIC_MAX_SPECIES];
    if ((rc = read_counters(8, g.ns, lost))) return rc;
    for (int s = 0; s < g.ns; ++s) {
      g.sp[s].n_live -= (int64_t)lost[s];
      if ((rc = zero_counter(8 + s))) return rc;
    }
  }
  // 4. MCC
  pic_mcc_stats ms;
  std::memset(&ms, 0, sizeof ms);
  if (g.mcc_ready)
    if ((rc = mcc_run(step, &ms, true))) return rc;
  PIC_CUDA(cudaStreamWaitEvent(g.st, e[9], 0));  // the fields are ready for the next push
  PIC_CUDA(cudaEventRecord(e[4], g.st));
  // 5. counting sort
  if ((int64_t)(step % (uint64_t)g.P.sort_interval) == 0)
    for (int s = 0; s < g.ns; ++s)
      if ((rc = sort_species(s))) return rc;
  PIC_CUDA(cudaEventRecord(e[5], g.st));
  // particles outside the mesh (counter 1) and push tiles that never
  // arrived (counter 2), one read (it also waits for the step)
  unsigned long long c12[2] = {0, 0};
  if ((rc = read_counters(1, 2, c12))) return rc;
  const unsigned long long bad = c12[0];
  if (c12[1]) {
    zero_counter(2);
    set_error("pic_step: a push tile copy did not complete within its bounded wait");
    return PIC_ERR_CUDA;
  }
  ++g.step_count;
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    for (int s = 0; s < g.ns; ++s) {
      stats->n_particles[s] = g.sp[s].n_live;
      stats->n_lost[s] = before[s] - g.sp[s].n_live + ms.n_created[s];
    }
    stats->solve = ss;
    stats->mcc = ms;
    float t;
    cudaEventElapsedTime(&t, e[0], e[1]); stats->ms_push = t;
    cudaEventElapsedTime(&t, e[1], e[2]); stats->ms_solve = t; stats->solve.ms = t;
    cudaEventElapsedTime(&t, e[8], e[9]); stats->ms_ppr = t;  // overlaps the MCC phase
    cudaEventElapsedTime(&t, e[3], e[4]); stats->ms_mcc = t;
    cudaEventElapsedTime(&t, e[4], e[5]); stats->ms_sort = t;
    cudaEventElapsedTime(&t, e[0], e[5]); stats->ms_total = t;
    cudaEventElapsedTime(&t, e[6], e[7]); stats->ms_push_kernel = t;
    stats->pushed = pushed;
  }
  if (bad) {
    set_error("pic_step: particle outside the mesh after the push");
    return PIC_ERR_DOMAIN;
  }
  return solve_rc;
}

int pic_get_fields_async(double *rho_out, double *phi_out, double *efx_out, double *efy_out) {
  int rc;
  if ((rc = check_init())) return rc;
  PIC_CUDA(cudaEventRecord(g.ev_copy_start, g.st));
  PIC_CUDA(cudaStreamWaitEvent(g.st_copy, g.ev_copy_start, 0));
  struct {
    double *host;
    const double *dev;
    int f;
  } c[4] = {{phi_out, g.d_phi, 1}, {rho_out, g.d_rho, 0}, {efx_out, g.d_efx, 2}, {efy_out, g.d_efy, 3}};
  for (auto &q : c) {
    if (!q.host) continue;
    PIC_CUDA(cudaMemcpyAsync(q.host, q.dev, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st_copy));
    PIC_CUDA(cudaEventRecord(g.ev_field[q.f], g.st_copy));
    g.copy_pending |= 1u << q.f;
  }
  return PIC_OK;
}

int pic_set_field_async(int32_t which, const double *host_in) {
  int rc;
  if ((rc = check_init())) return rc;
  if (!host_in || (which != 0 && which != 1)) {
    set_error("pic_set_field_async: which must be 0 (rho) or 1 (phi), host_in not NULL");
    return PIC_ERR_ARG;
  }
  double *dst = which == 0 ? g.d_rho : g.d_phi;
  // after what the library's stream has queued (the field may still be
  // read or written there) and after the copies already on the copy stream
  PIC_CUDA(cudaEventRecord(g.ev_copy_start, g.st));
  PIC_CUDA(cudaStreamWaitEvent(g.st_copy, g.ev_copy_start, 0));
  PIC_CUDA(cudaMemcpyAsync(dst, host_in, g.nn * sizeof(double), cudaMemcpyHostToDevice, g.st_copy));
  PIC_CUDA(cudaEventRecord(g.ev_field[which], g.st_copy));
  g.copy_pending |= 1u << which;
  return PIC_OK;
}

int pic_wait_fields(void) {
  int rc;
  if ((rc = check_init())) return rc;
  PIC_CUDA(cudaStreamSynchronize(g.st_copy));
  g.copy_pending = 0;
  return PIC_OK;
}

int pic_get_field(int32_t which, double *host_out) {
  int rc;
  if ((rc = check_init())) return rc;
  if (!host_out) return PIC_ERR_ARG;
  const double *src = nullptr;
  if (which == 0) src = g.d_rho;
  else if (which == 1) src = g.d_phi;
  else if (which == 2) src = g.d_efx;
  else if (which == 3) src = g.d_efy;
  else if (which >= 4 && which < 4 + g.ns) src = g.sp[which - 4].rho_s;
  else if (which >= 8 && which < 8 + g.ns) src = g.sp[which - 8].ek_s;
  else if (which >= 12 && which <= 16) src = g.d_coef + (size_t)(which - 12) * g.nn;
  else if (which == 20) src = g.d_b;
  else if (which >= 24 && which < 24 + g.ns) src = g.sp[which - 24].ek_tot;
  if (!src) {
    set_error("pic_get_field: unknown field");
    return PIC_ERR_ARG;
  }
  if ((rc = fields_fence(which <= 3 ? 1u << which : 0u))) return rc;  // an upload of it may be queued
  PIC_CUDA(cudaMemcpyAsync(host_out, src, g.nn * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  PIC_CUDA(cudaStreamSynchronize(g.st));
  return PIC_OK;
}

int pic_set_field(int32_t which, const double *host_in) {
  int rc;
  if ((rc = check_init())) return rc;
  if (!host_in) return PIC_ERR_ARG;
  double *dst = nullptr;
  if (which == 0) dst = g.d_rho;
  else if (which == 1) dst = g.d_phi;
  else if (which == 2) dst = g.d_efx;
  else if (which == 3) dst = g.d_efy;
  else if (which >= 12 && which <= 16) dst = g.d_coef + (size_t)(which - 12) * g.nn;
  if (!dst) {
    set_error("pic_set_field: unknown field");
    return PIC_ERR_ARG;
  }
  if ((rc = fields_fence(which <= 3 ? 1u << which : 0u))) return rc;
  PIC_CUDA(cudaMemcpyAsync(dst, host_in, g.nn * sizeof(double), cudaMemcpyHostToDevice, g.st));
  if (g.mixed && (which == 2 || which == 3 || which >= 12)) {
    k_coef32<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(g.d_efx, g.d_efy, g.d_coef, g.d_coef32, g.nn);
    PIC_LAUNCHED();
  }
  if (which == 2 || which == 3) {
    k_efxy<<<blocks_for(g.nn, 256), 256, 0, g.st>>>(g.d_efx, g.d_efy, g.d_efxy, g.nn);
    PIC_LAUNCHED();
  }
  PIC_CUDA(cudaStreamSynchronize(g.st));
  return PIC_OK;
}

}  // extern "C"
