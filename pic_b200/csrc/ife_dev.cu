// ife_dev.cu -- the interface elements' basis, stiffness and load matrix
// computed on the CUDA device in FP64, one thread per interface element,
// with the code of ife_elem.h that the host builder runs (so the device and
// host results are the same bits: --fmad=false here, -ffp-contract=off
// there).  pic_mesh_build_device takes its interface elements from here.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/picgpu.h"
#include "ife_elem.h"

namespace pic {
void set_error(const std::string &msg);

namespace {

__global__ void k_ife_elements(IfeElem *__restrict__ f, int n, int axi, double *__restrict__ K,
                               double *__restrict__ M, int *__restrict__ status) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  IfeElem e = f[k];
  status[k] = ife_element_all(e, axi, K + 16 * (size_t)k, M + 16 * (size_t)k);
  f[k] = e;  // with its basis coefficients
}

int dev_fail(cudaError_t e, const char *where) {
  set_error(std::string("pic_mesh_build_device: ") + where + ": " + cudaGetErrorString(e));
  return PIC_ERR_CUDA;
}

}  // namespace

// elems (host, n) in, their basis coefficients written back; K, M (host,
// 16 n) out.  Device memory is allocated for the call and freed after it.
int ife_elements_device(IfeElem *elems, int n, int axi, double *K, double *M) {
  IfeElem *df = nullptr;
  double *dk = nullptr, *dm = nullptr;
  int *ds = nullptr;
  int rc = PIC_OK;
  cudaError_t e;
  const size_t nm = 16 * (size_t)n;
  if ((e = cudaMalloc(&df, sizeof(IfeElem) * (size_t)n)) != cudaSuccess ||
      (e = cudaMalloc(&dk, sizeof(double) * nm)) != cudaSuccess ||
      (e = cudaMalloc(&dm, sizeof(double) * nm)) != cudaSuccess ||
      (e = cudaMalloc(&ds, sizeof(int) * (size_t)n)) != cudaSuccess) {
    rc = dev_fail(e, "cudaMalloc");
  } else if ((e = cudaMemcpy(df, elems, sizeof(IfeElem) * (size_t)n, cudaMemcpyHostToDevice)) != cudaSuccess) {
    rc = dev_fail(e, "copy in");
  } else {
    k_ife_elements<<<(n + 127) / 128, 128>>>(df, n, axi, dk, dm, ds);
    std::vector<int> st(n);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      rc = dev_fail(e, "launch");
    } else if ((e = cudaMemcpy(elems, df, sizeof(IfeElem) * (size_t)n, cudaMemcpyDeviceToHost)) != cudaSuccess ||
               (e = cudaMemcpy(K, dk, sizeof(double) * nm, cudaMemcpyDeviceToHost)) != cudaSuccess ||
               (e = cudaMemcpy(M, dm, sizeof(double) * nm, cudaMemcpyDeviceToHost)) != cudaSuccess ||
               (e = cudaMemcpy(st.data(), ds, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost)) != cudaSuccess) {
      rc = dev_fail(e, "copy out");
    } else {
      for (int k = 0; k < n; ++k)
        if (st[k]) {
          set_error(st[k] == 1 ? "pic_mesh_build_device: singular IFE basis system"
                               : "pic_mesh_build_device: singular interface load-matrix system");
          rc = PIC_ERR_SETUP;
          break;
        }
    }
  }
  cudaFree(df);
  cudaFree(dk);
  cudaFree(dm);
  cudaFree(ds);
  return rc;
}

}  // namespace pic
