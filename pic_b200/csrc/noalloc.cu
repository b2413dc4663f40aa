// noalloc.cu -- charge deposit of one species that allocates no memory.
//
// Some callers cannot allocate device memory: a host program whose memory
// pool is owned by another framework (for example a Fortran code whose
// device memory all comes from one pre-sized arena), a real-time loop that
// must not pay for the implicit device synchronisation of cudaMalloc, or a
// process that has already reserved the whole device.  pic_deposit_noalloc
// serves them: the caller passes its own input and output device buffers and
// the int64 fixed-point accumulator lives in a file-scope __device__ array
// of fixed size, so no call allocates or frees anything.
//
// The arithmetic is the one of the GetParChg_2D path of libpicgpu (locate,
// bilinear weights, 2^-40 fixed point with each particle depositing exactly
// 2^40, normalisation by the dual volume), so
// on a Cartesian mesh with FP64 positions the result equals pic_get_par_chg's
// per-species density bit for bit.  It has no r-z (delta 1) weighting and
// takes no FP32 element offsets (the mixed-precision particle layout).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "../../include/picgpu.h"
#include "pic_common.h"

namespace pic {
void set_error(const std::string &msg);
}

// Scratch: one int64 accumulator per mesh node, at most PIC_NOALLOC_MAX_NODES
// nodes (4 MiB).  Every device that loads the library holds it until exit.
static __device__ __align__(256) unsigned long long g_noalloc_acc[PIC_NOALLOC_MAX_NODES];

namespace {

constexpr int kMaxDevices = 64;
// Device address of g_noalloc_acc per device ordinal, looked up on the first
// call with that device current.  Atomic: host threads driving different
// devices may make their first calls at the same time.
std::atomic<unsigned long long *> g_acc_ptr[kMaxDevices];

__global__ void k_na_clear(unsigned long long *acc, int64_t nn) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) acc[i] = 0ull;
}

__global__ void k_na_deposit(int nnx, int nny, double xmin, double ymin, double hx, double hy, int64_t n,
                             const double *__restrict__ x, const double *__restrict__ y,
                             const int32_t *__restrict__ loc, unsigned long long *acc) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (loc && loc[p] < 0) return;  // absorbed slot
  const int nex = nnx - 1, ney = nny - 1;
  double px = x[p], py = y[p];
  double rxp = (px - xmin) / hx, ryp = (py - ymin) / hy;
  int i = (int)rxp + 1, j = (int)ryp + 1;
  if (i == nnx) i = nnx - 1;
  if (j == nny) j = nny - 1;
  if (!(rxp >= 0.0) || !(ryp >= 0.0) || i < 1 || j < 1 || i > nex || j > ney) return;
  int ie = i - 1, je = j - 1;
  double x1 = xmin + hx * ie, x2 = xmin + hx * (ie + 1);
  double y1 = ymin + hy * je, y2 = ymin + hy * (je + 1);
  double dx = (px - x1) / (x2 - x1);
  double dy = (py - y1) / (y2 - y1);
  double xc = 1.0 - dx, yc = 1.0 - dy;
  double W[4] = {xc * yc, dx * yc, dx * dy, xc * dy};
  int64_t n1 = (int64_t)ie * nny + je;
  int64_t nodes[4] = {n1, n1 + nny, n1 + nny + 1, n1 + 1};
  // corner 2 takes the rest of the particle's 2^40, as pic_get_par_chg does
  long long q[4];
  q[0] = __double2ll_rn(W[0] * PIC_Q_SCALE);
  q[1] = __double2ll_rn(W[1] * PIC_Q_SCALE);
  q[3] = __double2ll_rn(W[3] * PIC_Q_SCALE);
  q[2] = (1ll << 40) - ((q[0] + q[1]) + q[3]);
  for (int c = 0; c < 4; ++c) atomicAdd(acc + nodes[c], (unsigned long long)q[c]);
}

__global__ void k_na_normalize(const unsigned long long *acc, const double *__restrict__ vol, double wq,
                               double L_ref, double n_ref, double *__restrict__ rho, int64_t nn) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nn) return;
  double cnt = (double)(long long)acc[k] * (1.0 / PIC_Q_SCALE);
  rho[k] = ((((wq * cnt) / L_ref) / L_ref) / n_ref) / vol[k];
}

int na_fail(cudaError_t e, const char *where) {
  pic::set_error(std::string("pic_deposit_noalloc: ") + where + ": " + cudaGetErrorString(e));
  return PIC_ERR_CUDA;
}

}  // namespace

extern "C" int pic_deposit_noalloc(int32_t nnx, int32_t nny, double xmin, double xmax, double ymin,
                                   double ymax, int64_t n, const double *x, const double *y,
                                   const int32_t *loc, const double *cell_volume, double weight_charge,
                                   double L_ref, double n_ref, double *rho_out, void *stream) {
  if (nnx < 3 || nny < 3 || !(xmax > xmin) || !(ymax > ymin) || n < 0 || !cell_volume || !rho_out ||
      (n > 0 && (!x || !y)) || !(L_ref > 0) || !(n_ref > 0)) {
    pic::set_error("pic_deposit_noalloc: bad arguments");
    return PIC_ERR_ARG;
  }
  const int64_t nn = (int64_t)nnx * nny;
  if (nn > PIC_NOALLOC_MAX_NODES) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "pic_deposit_noalloc: mesh has %lld nodes, the static scratch holds at most %d",
             (long long)nn, PIC_NOALLOC_MAX_NODES);
    pic::set_error(buf);
    return PIC_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    pic::set_error("pic_deposit_noalloc: device ordinal beyond the supported range");
    return PIC_ERR_ARG;
  }
  // Set-up, once per device with that device current: the device address of
  // the scratch array (its host-side name is only a stand-in).
  unsigned long long *acc = g_acc_ptr[dev].load(std::memory_order_acquire);
  if (!acc) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_acc);
    if (e != cudaSuccess) return na_fail(e, "cudaGetSymbolAddress");
    acc = (unsigned long long *)ptr;
    g_acc_ptr[dev].store(acc, std::memory_order_release);
  }
  cudaStream_t st = (cudaStream_t)stream;
  const double hx = (xmax - xmin) / (nnx - 1), hy = (ymax - ymin) / (nny - 1);
  k_na_clear<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(acc, nn);
  if (n > 0)
    k_na_deposit<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nnx, nny, xmin, ymin, hx, hy, n, x, y, loc, acc);
  k_na_normalize<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(acc, cell_volume, weight_charge, L_ref, n_ref,
                                                                rho_out, nn);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(e, "launch");
  return PIC_OK;
}
