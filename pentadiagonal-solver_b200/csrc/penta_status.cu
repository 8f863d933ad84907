// penta_status.cu -- the status words kernels report into, and the bounded-wait
// self test.
//
// Status words live in a file-scope __device__ array of kStatusSlots words, so
// no solve ever allocates: every device that loads the library holds one copy
// of the array.  Slot 0 belongs to the handle-less calls (the reference's
// interface: one default context per device).  Every created handle and every
// plan takes a slot of its own from a free list, so the bits a kernel raises
// are attributed to the handle or plan that launched it, whatever stream it
// ran on; once the free list is empty, further handles and plans share slot 0
// (their status checks then also see the handle-less calls' bits).
//
// Reading is one kernel on the caller's stream, `*taken = atomicExch(word, 0)`,
// followed by a copy of `taken`: a bit a concurrent kernel ORs in is either in
// the value read or stays in the word for the next check -- never lost between
// a read and a separate clear.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "penta_internal.hpp"
#include "tma_device.cuh"

namespace {
__device__ int g_status_words[penta::kStatusSlots];
__device__ int g_status_taken[penta::kStatusSlots];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int *g_words[kMaxDevices] = {};
int *g_taken[kMaxDevices] = {};
std::vector<int> g_free;  // free slots (1 .. kStatusSlots-1), filled on first use
bool g_free_init = false;

bool addresses(int device) {  // caller holds g_mu
  if (g_words[device] != nullptr) return true;
  void *w = nullptr, *t = nullptr;
  if (cudaGetSymbolAddress(&w, g_status_words) != cudaSuccess ||
      cudaGetSymbolAddress(&t, g_status_taken) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  g_words[device] = static_cast<int *>(w);
  g_taken[device] = static_cast<int *>(t);
  return true;
}

__global__ void status_take_kernel(int *word, int *taken) {
  if (threadIdx.x == 0) *taken = atomicExch(word, 0);
}

// The bounded-wait self test: thread 0 initialises an mbarrier that expects
// two arrivals and arrives once, so the phase never completes; the wait gives
// up after `limit_ns` of %globaltimer and the kernel raises STATUS_TIMEOUT_BIT,
// exactly as the solvers do when one of their waits runs out.
__global__ void bounded_wait_selftest_kernel(unsigned long long limit_ns, int *status_word) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    penta::mbar_init(&bar, 2);
    penta::mbar_init_fence();
    penta::mbar_arrive(&bar);
    if (!penta::mbar_wait_for(&bar, 0u, limit_ns)) atomicOr(status_word, penta::STATUS_TIMEOUT_BIT);
  }
}
}  // namespace

namespace penta {

int *status_word(int device, int slot) {
  if (device < 0 || device >= kMaxDevices || slot < 0 || slot >= kStatusSlots) return nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!addresses(device)) return nullptr;
  return g_words[device] + slot;
}

int *device_status_word(int device) { return status_word(device, 0); }

int status_slot_acquire() {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_free_init) {
    for (int s = kStatusSlots - 1; s >= 1; --s) g_free.push_back(s);
    g_free_init = true;
  }
  if (g_free.empty()) return 0;  // shared with the handle-less calls
  const int s = g_free.back();
  g_free.pop_back();
  return s;
}

void status_slot_release(int slot, int device) {
  if (slot <= 0 || slot >= kStatusSlots) return;
  if (device >= 0 && device < kMaxDevices) {
    // clear what the owner left unread, so the next owner starts at zero
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess) {
      if (cur != device) cudaSetDevice(device);
      const int zero = 0;
      if (cudaMemcpyToSymbol(g_status_words, &zero, sizeof(int), slot * sizeof(int),
                             cudaMemcpyHostToDevice) != cudaSuccess)
        cudaGetLastError();
      if (cur != device) cudaSetDevice(cur);
    } else {
      cudaGetLastError();
    }
  }
  std::lock_guard<std::mutex> lock(g_mu);
  g_free.push_back(slot);
}

cudaError_t status_take(int device, int slot, cudaStream_t stream, int *bits) {
  int *word = status_word(device, slot);
  if (word == nullptr) return cudaErrorInvalidValue;
  int *taken;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    taken = g_taken[device] + slot;
  }
  status_take_kernel<<<1, 32, 0, stream>>>(word, taken);
  cudaError_t e = cudaGetLastError();
  int host = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&host, taken, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && bits != nullptr) *bits = host;
  return e;
}

cudaError_t launch_bounded_wait_selftest(unsigned long long limit_ns, int *status,
                                         cudaStream_t stream) {
  bounded_wait_selftest_kernel<<<1, 32, 0, stream>>>(limit_ns, status);
  return cudaGetLastError();
}

}  // namespace penta
