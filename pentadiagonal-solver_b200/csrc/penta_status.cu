// penta_status.cu -- the per-device status word kernels report into.
//
// A file-scope __device__ word: every device that loads the library gets one,
// so no solve ever allocates.  Kernels OR status bits (penta_device.cuh) into
// it; pentadsolver_status_check reads and clears it.
#include <cuda_runtime.h>

#include <mutex>

#include "penta_internal.hpp"

namespace {
__device__ int g_status_word;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int *g_addr[kMaxDevices] = {};
}  // namespace

namespace penta {

int *device_status_word(int device) {
  if (device < 0 || device >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[device] == nullptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_status_word) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_addr[device] = static_cast<int *>(p);
  }
  return g_addr[device];
}

}  // namespace penta
