// penta_api.cpp -- the C ABI and the host-side dispatcher.
//
// Entry points keep the reference's names and argument meaning
// (include/pentadsolver.hpp, include/pentadsolver_cuda.hpp); the routing
// follows the reference's router src/cuda/singlenode/pentad_cuda.cu:1512-1540:
// solvedim 0 -> x, solvedim t_ndim-1 -> outermost, otherwise middle.  Each
// direction then picks a kernel family from the PENTA_*ALGO selectors
// (pentad_cuda.cu:1163-1174 for y/z, :1463-1489 for x), the handle's own
// choice, or the automatic choice, and records what it launched.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdint>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "pentad_common.hpp"
#include "pentadsolver.hpp"
#include "pentadsolver_ext.h"
#include "penta_internal.hpp"

namespace penta {
namespace {

constexpr int kMaxDevices = 64;
constexpr const char *kNone = "none";

enum class Algo { Auto, Naive, Transpose, ThomasPcr, SharedFact, Unknown };

const char *algo_name(Algo a) {
  switch (a) {
    case Algo::Naive: return "naive";
    case Algo::Transpose: return "transpose";
    case Algo::ThomasPcr: return "thomas-pcr";
    case Algo::SharedFact: return "shared-fact";
    case Algo::Auto: return "auto";
    default: return "unknown";
  }
}

Algo parse_algo(const char *s) {
  if (s == nullptr || s[0] == '\0') return Algo::Auto;
  if (!std::strcmp(s, "auto")) return Algo::Auto;
  if (!std::strcmp(s, "naive") || !std::strcmp(s, "legacy")) return Algo::Naive;
  if (!std::strcmp(s, "transpose")) return Algo::Transpose;
  if (!std::strcmp(s, "thomas-pcr")) return Algo::ThomasPcr;
  if (!std::strcmp(s, "shared-fact")) return Algo::SharedFact;
  return Algo::Unknown;
}

bool env_flag(const char *name) {
  const char *v = std::getenv(name);
  return v != nullptr && v[0] == '1';
}

// Kernel-choice knobs for one solve: the handle's tuning for the direction
// (pentadsolver_set_tuning: "auto", "no-tmem", "no-tma", "tmem=ST,XST",
// "tma=R,ST,XST,SCR") when set, else the PENTA_NO_TMEM / PENTA_NO_TMA /
// PENTA_TMEM_VARIANT / PENTA_TMA_VARIANT environment variables.
struct Knobs {
  bool no_tma = false, no_tmem = false;
  std::string tmem_variant, tma_variant;
};
Knobs knobs_from(const std::string &tuning) {
  Knobs k;
  if (!tuning.empty()) {
    if (tuning == "no-tma") k.no_tma = true;
    else if (tuning == "no-tmem") k.no_tmem = true;
    else if (tuning.rfind("tmem=", 0) == 0) k.tmem_variant = tuning.substr(5);
    else if (tuning.rfind("tma=", 0) == 0) {
      k.no_tmem = true;
      k.tma_variant = tuning.substr(4);
    }
    return k;
  }
  k.no_tma = env_flag("PENTA_NO_TMA");
  k.no_tmem = env_flag("PENTA_NO_TMEM");
  if (const char *e = std::getenv("PENTA_TMEM_VARIANT")) k.tmem_variant = e;
  if (const char *e = std::getenv("PENTA_TMA_VARIANT")) k.tma_variant = e;
  return k;
}

// Does the environment fix the kernel choice of this direction (the algorithm
// selectors, PENTA_PCR_LANES, or a kernel knob)?  Then the tuning table is
// not consulted, as the reference's selectors win over everything.
bool env_fixes_choice(int dir) {
  auto set = [](const char *name) {
    const char *v = std::getenv(name);
    return v != nullptr && v[0] != '\0';
  };
  if (dir == 0 ? set("PENTA_XALGO")
               : (set(dir == 1 ? "PENTA_YALGO" : "PENTA_ZALGO") || set("PENTA_YZALGO")))
    return true;
  return set("PENTA_PCR_LANES") || env_flag("PENTA_NO_TMA") || env_flag("PENTA_NO_TMEM") ||
         set("PENTA_TMEM_VARIANT") || set("PENTA_TMA_VARIANT");
}

// ---------------------------------------------------------------------------
// Contexts
// ---------------------------------------------------------------------------
struct Context {
  int device = -1;
  int slot = 0;  // status word slot (0: shared by the handle-less calls)
  int sm_count = 0;
  int smem_optin = 0;  // max dynamic shared memory per block (bytes)
  std::mutex mu;
  Algo forced[3] = {Algo::Auto, Algo::Auto, Algo::Auto};
  int forced_lanes[3] = {0, 0, 0};
  std::atomic<const char *> ran[3] = {{kNone}, {kNone}, {kNone}};
  std::string variant[3];
  std::string tuning[3];  // pentadsolver_set_tuning, per direction ("" = none)
  std::unordered_map<long long, int> occ_cache;  // (variant, n) -> CTAs/SM
  std::string gpu_name;  // the device's name (tuning-table keys)
  cudaStream_t copy_stream = nullptr;  // non-blocking: plan-table uploads (copy_h2d)

  bool init() {  // idempotent; needs a usable device
    if (device >= 0) return true;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    int sms = 0, optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                               dev) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    gpu_name = prop.name;
    sm_count = sms;
    smem_optin = optin;
    device = dev;
    return true;
  }
};

// Host -> device copy that waits only for itself: on the context's
// non-blocking stream, so creating a plan never waits for solves that run on
// other streams (a plain cudaMemcpy on the legacy stream can).
cudaError_t copy_h2d(Context &ctx, void *dst, const void *src, size_t bytes) {
  cudaStream_t s = nullptr;
  {
    std::lock_guard<std::mutex> lock(ctx.mu);
    if (ctx.copy_stream == nullptr &&
        cudaStreamCreateWithFlags(&ctx.copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
      ctx.copy_stream = nullptr;
      return cudaGetLastError();
    }
    s = ctx.copy_stream;
  }
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

std::mutex g_reg_mu;
std::unordered_set<Context *> g_live;
Context *g_default[kMaxDevices] = {};
std::atomic<const char *> g_ran[3] = {{kNone}, {kNone}, {kNone}};

// A created handle, or the default context of the current device.
Context *resolve(pentadsolver_handle_t h) {
  std::lock_guard<std::mutex> lock(g_reg_mu);
  if (h != nullptr) {
    auto *c = static_cast<Context *>(h);
    if (g_live.count(c)) return c;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  if (dev < 0 || dev >= kMaxDevices) dev = 0;
  if (g_default[dev] == nullptr) g_default[dev] = new Context();
  return g_default[dev];
}

// ---------------------------------------------------------------------------
// Shapes and buffer layout
// ---------------------------------------------------------------------------
struct Shape {
  Lines L{};
  int dir = 0;  // 0 x, 1 middle, 2 outermost
};

pentadStatus_t make_shape(const int *dims, int ndim, int solvedim, Shape &sh,
                          const char **why) {
  if (dims == nullptr) { *why = "t_dims is null"; return PENTAD_STATUS_INVALID_VALUE; }
  if (ndim < 1 || ndim > PENTAD_MAXDIM) {
    *why = "t_ndim out of range [1, 8]";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (solvedim < 0 || solvedim >= ndim) {
    *why = "t_solvedim out of range";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  // products are checked before they are formed: no overflow whatever the dims
  constexpr long long kMaxSystems = 1LL << 40;
  long long inner = 1, systems = 1;
  for (int k = 0; k < ndim; ++k) {
    if (dims[k] < 1) { *why = "a dimension is < 1"; return PENTAD_STATUS_INVALID_VALUE; }
    if (k == solvedim) continue;
    if (systems > kMaxSystems / dims[k]) {
      *why = "grid too large";
      return PENTAD_STATUS_INVALID_VALUE;
    }
    systems *= dims[k];
    if (k < solvedim) inner *= dims[k];
  }
  const long long n = dims[solvedim];
  if (n <= 4) {
    // The reference asserts sys_size > 4 on every path (pentad_cuda.cu:1203).
    *why = "the solve dimension must be longer than 4";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (n > (1LL << 24)) {
    *why = "grid too large";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  sh.L.n = n;
  sh.L.inner = inner;
  sh.L.n_sys = systems;
  sh.dir = (solvedim == 0) ? 0 : (solvedim == ndim - 1 ? 2 : 1);
  return PENTAD_STATUS_SUCCESS;
}

// The reference's sizing (src/cuda/singlenode/pentad_cuda.cu:1554-1577): 9 n
// n_sys elements along x (room for its transpose path), 3 n n_sys otherwise.
// Every kernel here fits in that: the global-scratch Thomas kernel uses the
// first 3 n n_sys elements, the on-chip kernels less.
size_t buffer_bytes(const Shape &sh, size_t elem) {
  const size_t regions = (sh.dir == 0) ? 9 : 3;
  return regions * (size_t)sh.L.n * (size_t)sh.L.n_sys * elem;
}

// ---------------------------------------------------------------------------
// Selection
// ---------------------------------------------------------------------------
Algo selected_algo(Context &ctx, int dir) {
  if (dir == 0) {
    const char *e = std::getenv("PENTA_XALGO");
    if (e != nullptr && e[0] != '\0') {
      Algo a = parse_algo(e);
      // unknown x selectors fall through to auto (pentad_cuda.cu:1457-1461)
      return a == Algo::Unknown ? Algo::Auto : a;
    }
  } else {
    const char *e = std::getenv(dir == 1 ? "PENTA_YALGO" : "PENTA_ZALGO");
    if (e == nullptr || e[0] == '\0') e = std::getenv("PENTA_YZALGO");
    if (e != nullptr && e[0] != '\0') {
      Algo a = parse_algo(e);
      // unknown y/z selectors mean the legacy kernel (pentad_cuda.cu:1143-1152);
      // "transpose" has no strided meaning either
      if (a == Algo::Unknown || a == Algo::Transpose) return Algo::Naive;
      return a;
    }
  }
  return ctx.forced[dir];
}

int selected_lanes(Context &ctx, int dir) {
  if (const char *e = std::getenv("PENTA_PCR_LANES")) {
    const int v = std::atoi(e);
    if (v == 1 || v == 2 || v == 4 || v == 8 || v == 16 || v == 32) return v;
  }
  return ctx.forced_lanes[dir];
}

// The on-chip (tiled) variant for a shape: among the compiled variants of
// this precision, layout and partition count whose shared memory fits, the
// one with the most resident CTAs per SM (capped at 4), then the deepest
// ring.  Occupancy queries are cached per (variant, n).
template <typename F>
bool pick_tiled(Context &ctx, const Lines &L, bool contig, int P,
                TiledConfig &out, int &occ_out) {
  if (L.n * L.n_sys >= (1LL << 31)) return false;  // 32-bit in-tile offsets
  const std::vector<TiledConfig> &all = tiled2_configs<F>();
  int best = -1, best_score = -1, best_occ = 0;
  for (size_t i = 0; i < all.size(); ++i) {
    const TiledConfig &c = all[i];
    if (c.contig != contig || (P != 0 && c.P != P)) continue;
    if (tiled2_smem_bytes<F>(c, L.n) > (size_t)ctx.smem_optin) continue;
    int occ;
    const long long key = ((long long)i << 40) | (L.n << 1) | (sizeof(F) == 8);
    {
      std::lock_guard<std::mutex> lock(ctx.mu);
      auto it = ctx.occ_cache.find(key);
      occ = (it != ctx.occ_cache.end()) ? it->second : -1;
    }
    if (occ < 0) {
      occ = tiled2_occupancy<F>(c, L.n);
      std::lock_guard<std::mutex> lock(ctx.mu);
      ctx.occ_cache[key] = occ;
    }
    if (occ <= 0) continue;
    const int score = std::min(occ, 4) * 1000 + c.stages * c.R;
    if (score > best_score) {
      best_score = score;
      best = (int)i;
      best_occ = occ;
    }
  }
  if (best < 0) return false;
  out = all[best];
  occ_out = best_occ;
  return true;
}

// The TMA-fed strided variant: most resident CTAs (capped at 4), then the
// deepest ring.
template <typename F>
bool pick_tma(Context &ctx, const SolveArgs<F> &a, size_t usable_buf, TmaConfig &out,
              int &occ_out, const std::string &variant) {
  if (!tma_supported<F>(a)) return false;
  // the scratch variants keep (dw2, x2) in the caller's buffer
  // (128-byte aligned: they drop whole 128-byte lines of it from L2)
  const bool scr_ok = a.scratch != nullptr &&
                      reinterpret_cast<uintptr_t>(a.scratch) % 128 == 0 &&
                      tma_scratch_bytes<F>(a.L) <= usable_buf;
  const std::vector<TmaConfig> &all = tma_configs<F>();
  // "R,stages,xstages,scratch" restricts the choice (tuning)
  int want[4] = {-1, -1, -1, -1};
  if (!variant.empty())
    std::sscanf(variant.c_str(), "%d,%d,%d,%d", &want[0], &want[1], &want[2], &want[3]);
  int best = -1, best_score = -1, best_occ = 0;
  for (size_t i = 0; i < all.size(); ++i) {
    const TmaConfig &c = all[i];
    if (c.scratch && !scr_ok) continue;
    if ((want[0] >= 0 && c.R != want[0]) || (want[1] >= 0 && c.stages != want[1]) ||
        (want[2] >= 0 && c.xstages != want[2]) ||
        (want[3] >= 0 && (int)c.scratch != want[3]))
      continue;
    if (tma_smem_bytes<F>(c, a.L.n) > (size_t)ctx.smem_optin) continue;
    int occ;
    const long long key =
        (1LL << 62) | ((long long)i << 40) | (a.L.n << 1) | (sizeof(F) == 8);
    {
      std::lock_guard<std::mutex> lock(ctx.mu);
      auto it = ctx.occ_cache.find(key);
      occ = (it != ctx.occ_cache.end()) ? it->second : -1;
    }
    if (occ < 0) {
      occ = tma_occupancy<F>(c, a.L.n);
      std::lock_guard<std::mutex> lock(ctx.mu);
      ctx.occ_cache[key] = occ;
    }
    if (occ <= 0) continue;
    const int score = std::min(occ, 4) * 1000 + c.stages * c.R;
    if (score > best_score) {
      best_score = score;
      best = (int)i;
      best_occ = occ;
    }
  }
  if (best < 0) return false;
  out = all[best];
  occ_out = best_occ;
  return true;
}

// The TMA-fed contiguous (x) variant: most resident CTAs (capped at 4), then
// the deepest ring.  It needs the caller's buffer for (dw2, x2).
template <typename F>
bool pick_tma_contig(Context &ctx, const SolveArgs<F> &a, size_t usable_buf,
                     TmaConfig &out, int &occ_out) {
  if (!tma_contig_supported<F>(a) || tma_contig_scratch_bytes<F>(a.L) > usable_buf)
    return false;
  const std::vector<TmaConfig> &all = tma_contig_configs<F>();
  int best = -1, best_score = -1, best_occ = 0;
  for (size_t i = 0; i < all.size(); ++i) {
    const TmaConfig &c = all[i];
    if (tma_contig_smem_bytes<F>(c, a.L.n) > (size_t)ctx.smem_optin) continue;
    int occ;
    const long long key =
        (1LL << 61) | ((long long)i << 40) | (a.L.n << 1) | (sizeof(F) == 8);
    {
      std::lock_guard<std::mutex> lock(ctx.mu);
      auto it = ctx.occ_cache.find(key);
      occ = (it != ctx.occ_cache.end()) ? it->second : -1;
    }
    if (occ < 0) {
      occ = tma_contig_occupancy<F>(c, a.L.n);
      std::lock_guard<std::mutex> lock(ctx.mu);
      ctx.occ_cache[key] = occ;
    }
    if (occ <= 0) continue;
    const int score = std::min(occ, 4) * 1000 + c.stages;
    if (score > best_score) {
      best_score = score;
      best = (int)i;
      best_occ = occ;
    }
  }
  if (best < 0) return false;
  out = all[best];
  occ_out = best_occ;
  return true;
}

// The Tensor-Memory kernel: the first compiled variant of this precision and
// layout that fits shared memory and runs one CTA per SM.
// "stages,xstages" restricts the choice (tuning).
template <typename F>
bool pick_tmem(Context &ctx, const SolveArgs<F> &a, bool contig, size_t usable_buf,
               TmemConfig &out, const std::string &variant) {
  int fmode = 0;
  if (!tmem_supported<F>(a, contig, usable_buf, fmode)) return false;
  const int loads = tmem_loads<F>(a, contig);
  int want[2] = {-1, -1};
  if (!variant.empty()) std::sscanf(variant.c_str(), "%d,%d", &want[0], &want[1]);
  const std::vector<TmemConfig> &all = tmem_configs<F>();
  for (size_t i = 0; i < all.size(); ++i) {
    const TmemConfig &c = all[i];
    if (c.contig != contig || c.fmode != fmode || c.loads != loads) continue;
    // factor mode 3 reads nothing back: only the ring depth of a choice applies
    if ((want[0] >= 0 && c.stages != want[0]) ||
        (want[1] >= 0 && fmode != 3 && c.xstages != want[1]))
      continue;
    if (c.smem > (size_t)ctx.smem_optin) continue;
    int occ;
    const long long key = (1LL << 59) | ((long long)i << 1) | (sizeof(F) == 8);
    {
      std::lock_guard<std::mutex> lock(ctx.mu);
      auto it = ctx.occ_cache.find(key);
      occ = (it != ctx.occ_cache.end()) ? it->second : -1;
    }
    if (occ < 0) {
      occ = tmem_occupancy<F>(c);
      std::lock_guard<std::mutex> lock(ctx.mu);
      ctx.occ_cache[key] = occ;
    }
    if (occ == 1) {  // exactly one CTA per SM: it owns all of Tensor Memory
      out = c;
      return true;
    }
  }
  return false;
}

std::string tiled_variant_name(const TiledConfig &c) {
  char buf[96];
  std::snprintf(buf, sizeof buf, "thomas-pcr:tiled P%d S%d R%d x%d%s", c.P,
                c.S, c.R, c.stages, c.contig ? " contig" : "");
  return buf;
}

void record(Context &ctx, int dir, const char *family, const std::string &var) {
  ctx.ran[dir].store(family);
  g_ran[dir].store(family);
  std::lock_guard<std::mutex> lock(ctx.mu);
  ctx.variant[dir] = var;
}

// ---------------------------------------------------------------------------
// The solve
// ---------------------------------------------------------------------------
// The context's device must be current: its cached device properties and its
// status word's address belong to that device.
bool on_own_device(const Context &ctx, const char **why) {
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) {
    cudaGetLastError();
    *why = "no usable CUDA device";
    return false;
  }
  if (cur != ctx.device) {
    *why = "the handle is bound to another device than the current one";
    return false;
  }
  return true;
}

// `slot` >= 0 reports into that status slot instead of the context's own
// (a plan's grids solved one by one).
template <typename F>
pentadStatus_t solve(Context &ctx, const F *ds, const F *dl, const F *d,
                     const F *du, const F *dw, F *x, const int *dims,
                     int ndim, int solvedim, void *buf, size_t buf_bytes,
                     cudaStream_t stream, const char **why, int slot = -1) {
  Shape sh;
  pentadStatus_t st = make_shape(dims, ndim, solvedim, sh, why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (!ds || !dl || !d || !du || !dw || !x) {
    *why = "an array pointer is null";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (!ctx.init()) {
    *why = "no usable CUDA device";
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  if (!on_own_device(ctx, why)) return PENTAD_STATUS_INVALID_VALUE;
  int *status_word = penta::status_word(ctx.device, slot >= 0 ? slot : ctx.slot);
  if (status_word == nullptr) {
    *why = "cannot address the device status word";
    return PENTAD_STATUS_INTERNAL_ERROR;
  }
  SolveArgs<F> a{ds, dl, d, du, dw, x, sh.L, buf, buf_bytes, status_word};
  const int dir = sh.dir;
  const bool contig = (dir == 0);
  Algo want = selected_algo(ctx, dir);
  int lanes = selected_lanes(ctx, dir);
  Knobs kn;
  bool open_choice;
  {
    std::lock_guard<std::mutex> lock(ctx.mu);
    kn = knobs_from(ctx.tuning[dir]);
    open_choice = ctx.tuning[dir].empty() && ctx.forced[dir] == Algo::Auto &&
                  ctx.forced_lanes[dir] == 0;
  }
  // the tuning table decides what neither the environment nor the handle fixes
  if (open_choice && !tune_table_empty() && !env_fixes_choice(dir)) {
    TuneChoice tc;
    if (tune_lookup(tune_key(ctx.gpu_name, "solve", sizeof(F), dir, sh.L.n, sh.L.n_sys), tc)) {
      kn = knobs_from(tc.spec.empty() ? std::string("auto") : tc.spec);
      const Algo ta = parse_algo(tc.algo.c_str());
      want = ta == Algo::Unknown ? Algo::Auto : ta;
      lanes = tc.lanes;
    }
  }
  const bool debug = env_flag("PENTA_DEBUG_LAUNCH");

  cudaError_t err = cudaSuccess;
  auto run_naive = [&]() -> pentadStatus_t {
    const size_t need = thomas_global_scratch<F>(sh.L);
    if (buf == nullptr || buf_bytes < need) {
      *why = "the naive kernel needs t_buffer of buffer_size_ext bytes";
      return PENTAD_STATUS_INVALID_VALUE;
    }
    err = launch_thomas_global<F>(a, stream);
    if (err != cudaSuccess) return PENTAD_STATUS_EXECUTION_FAILED;
    record(ctx, dir, "naive", "naive:global-scratch");
    return PENTAD_STATUS_SUCCESS;
  };
  auto run_tiled = [&](int P, const char *family) -> int {
    TiledConfig cfg{};
    int occ = 0;
    if (!pick_tiled<F>(ctx, sh.L, contig, P, cfg, occ)) return 0;  // declined
    err = launch_tiled2<F>(a, cfg, occ * ctx.sm_count, stream);
    if (err != cudaSuccess) {
      if (debug)
        std::fprintf(stderr, "[penta] %s launch declined: %s -- falling back\n",
                     tiled_variant_name(cfg).c_str(), cudaGetErrorString(err));
      cudaGetLastError();
      return 0;
    }
    std::string var = tiled_variant_name(cfg);
    if (!std::strcmp(family, "transpose")) var = "transpose:" + var.substr(11);
    record(ctx, dir, family, var);
    return 1;
  };

  switch (want) {
    case Algo::Naive:
      return run_naive();
    case Algo::Transpose:  // x only: on-chip transpose, one thread per system
      if (run_tiled(1, "transpose")) return PENTAD_STATUS_SUCCESS;
      break;
    case Algo::SharedFact: {  // line 0's coefficients for every line (not checked)
      const size_t usable = buf ? std::min(buf_bytes, buffer_bytes(sh, sizeof(F))) : 0;
      if (!kn.no_tma && sf_tmem_supported<F>(a, contig, ctx.smem_optin)) {
        int occ;
        const long long key = (1LL << 58) | ((long long)contig << 1) | (sizeof(F) == 8);
        {
          std::lock_guard<std::mutex> lock(ctx.mu);
          auto it = ctx.occ_cache.find(key);
          occ = (it != ctx.occ_cache.end()) ? it->second : -1;
        }
        if (occ < 0) {
          occ = sf_tmem_occupancy<F>(contig);
          std::lock_guard<std::mutex> lock(ctx.mu);
          ctx.occ_cache[key] = occ;
        }
        if (occ == 1) {  // one CTA per SM: it owns all of Tensor Memory
          err = launch_sf_tmem<F>(a, contig, ctx.sm_count, usable, stream);
          if (err == cudaSuccess) {
            record(ctx, dir, "shared-fact",
                   contig ? "shared-fact:tmem S32 contig" : "shared-fact:tmem S32");
            return PENTAD_STATUS_SUCCESS;
          }
          if (debug)
            std::fprintf(stderr, "[penta] shared-fact tmem launch declined: %s\n",
                         cudaGetErrorString(err));
          cudaGetLastError();
        }
      }
      if (usable < sf_lines_scratch_bytes<F>(sh.L)) {
        *why = "shared-fact needs t_buffer of buffer_size_ext bytes for this shape";
        return PENTAD_STATUS_INVALID_VALUE;
      }
      err = launch_sf_lines<F>(a, stream);
      if (err != cudaSuccess) return PENTAD_STATUS_EXECUTION_FAILED;
      record(ctx, dir, "shared-fact", "shared-fact:lines");
      return PENTAD_STATUS_SUCCESS;
    }
    case Algo::ThomasPcr:
    case Algo::Auto:
    default: {
      const int P = (lanes == 1) ? 1 : 2;
      if (P == 2 && !kn.no_tma && !kn.no_tmem) {
        TmemConfig mc{};
        const size_t usable = std::min(buf_bytes, buffer_bytes(sh, sizeof(F)));
        if (pick_tmem<F>(ctx, a, contig, usable, mc, kn.tmem_variant)) {
          err = launch_tmem<F>(a, mc, ctx.sm_count, stream);
          if (err == cudaSuccess) {
            char vb[96];
            const char *ld = mc.loads == 1 ? tmem_loader<F>(a, contig) : "";
            std::snprintf(vb, sizeof vb, "thomas-pcr:tmem P2 S16 R%d x%d/%d%s%s%s", mc.R,
                          mc.stages, mc.xstages,
                          mc.fmode == 2   ? " fbuf"
                          : mc.fmode == 1 ? " w2s"
                          : mc.fmode == 3 ? " x2t"
                                          : "",
                          ld,
                          contig ? " contig" : "");
            record(ctx, dir, "thomas-pcr", vb);
            return PENTAD_STATUS_SUCCESS;
          }
          if (debug)
            std::fprintf(stderr, "[penta] tmem launch declined: %s -- falling back\n",
                         cudaGetErrorString(err));
          cudaGetLastError();
        }
      }
      if (contig && P == 2 && !kn.no_tma) {
        TmaConfig tc{};
        int occ = 0;
        const size_t usable = std::min(buf_bytes, buffer_bytes(sh, sizeof(F)));
        if (pick_tma_contig<F>(ctx, a, usable, tc, occ)) {
          err = launch_tma_contig<F>(a, tc, occ * ctx.sm_count, stream);
          if (err == cudaSuccess) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "thomas-pcr:tma P2 S16 R%d x%d/%d contig",
                          tc.R, tc.stages, tc.xstages);
            record(ctx, dir, "thomas-pcr", buf);
            return PENTAD_STATUS_SUCCESS;
          }
          if (debug)
            std::fprintf(stderr, "[penta] tma launch declined: %s -- falling back\n",
                         cudaGetErrorString(err));
          cudaGetLastError();
        }
      }
      if (!contig && P == 2 && !kn.no_tma) {
        TmaConfig tc{};
        int occ = 0;
        const size_t usable = std::min(buf_bytes, buffer_bytes(sh, sizeof(F)));
        if (pick_tma<F>(ctx, a, usable, tc, occ, kn.tma_variant)) {
          err = launch_tma<F>(a, tc, occ * ctx.sm_count, stream);
          if (err == cudaSuccess) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "thomas-pcr:tma P2 S16 R%d x%d/%d%s",
                          tc.R, tc.stages, tc.xstages, tc.scratch ? " scr" : "");
            record(ctx, dir, "thomas-pcr", buf);
            return PENTAD_STATUS_SUCCESS;
          }
          if (debug)
            std::fprintf(stderr, "[penta] tma launch declined: %s -- falling back\n",
                         cudaGetErrorString(err));
          cudaGetLastError();
        }
      }
      if (run_tiled(P, "thomas-pcr")) return PENTAD_STATUS_SUCCESS;
      if (P == 1 && run_tiled(2, "thomas-pcr")) return PENTAD_STATUS_SUCCESS;
      break;
    }
  }
  if (debug)
    std::fprintf(stderr, "[penta] dir %d: %s not available for n=%lld, using naive\n",
                 dir, algo_name(want), sh.L.n);
  return run_naive();
}

template <typename F>
void solve_void(pentadsolver_handle_t h, const F *ds, const F *dl, const F *d,
                const F *du, const F *dw, F *x, const int *dims, int ndim,
                int solvedim, void *buf) {
  Context *ctx = resolve(h);
  const char *why = "";
  pentadStatus_t st = solve<F>(*ctx, ds, dl, d, du, dw, x, dims, ndim,
                               solvedim, buf, SIZE_MAX, (cudaStream_t)0, &why);
  if (st != PENTAD_STATUS_SUCCESS) {
    cudaError_t e = cudaGetLastError();
    std::fprintf(stderr, "[penta] solvedim %d launch FAILED: %s%s%s -- output is invalid\n",
                 solvedim, why, e != cudaSuccess ? ": " : "",
                 e != cudaSuccess ? cudaGetErrorString(e) : "");
  }
}

template <typename F>
pentadStatus_t solve_ex(pentadsolver_handle_t h, const F *ds, const F *dl,
                        const F *d, const F *du, const F *dw, F *x,
                        const int *dims, int ndim, int solvedim, void *buf,
                        size_t buf_bytes, void *stream) {
  Context *ctx = resolve(h);
  const char *why = "";
  pentadStatus_t st =
      solve<F>(*ctx, ds, dl, d, du, dw, x, dims, ndim, solvedim, buf,
               buf_bytes, static_cast<cudaStream_t>(stream), &why);
  if (st != PENTAD_STATUS_SUCCESS && env_flag("PENTA_DEBUG_LAUNCH"))
    std::fprintf(stderr, "[penta] solve rejected: %s\n", why);
  if (st == PENTAD_STATUS_EXECUTION_FAILED) cudaGetLastError();
  return st;
}

// ---------------------------------------------------------------------------
// Plans: many grids solved along one solvedim in one persistent launch
// ---------------------------------------------------------------------------
size_t round256(size_t v) { return (v + 255) & ~size_t(255); }

struct PlanSingle {  // a grid the batched kernel does not take: solved alone
  pentadsolver_grid_t g;
  size_t offset, bytes;
};

struct Plan {
  Context *ctx = nullptr;
  int slot = 0;  // status word slot of this plan
  std::string tkey;  // its tuning-table key (longest line, all lines)
  int elem = 8, solvedim = 0;
  bool contig = false, w2s = false, discard = false;
  unsigned char *table = nullptr, *scratch = nullptr;
  int n_jobs = 0, total_tiles = 0, ctas = 0;
  struct Group {  // one batched launch: jobs [first, first + count) of the table
    int first, count, tiles;
    int fmode;  // factor mode of its grids
    int loads;  // their stage layout (TMA tiles / bulk copies)
  };
  std::vector<Group> groups;
  std::vector<PlanSingle> singles;
  std::string desc;
  // mixed-precision refinement over the same grids (refine plans only)
  bool refine = false;
  int steps = 0, chunks = 0;
  RefineGrid *rtable = nullptr;  // device
  double *est = nullptr;         // device [count][2]
  int count = 0;
  Plan *fp32 = nullptr;          // the FP32 plan over the cast copies
  Plan *fp32q = nullptr;         // the same over the q arrays (one-step form)
  bool cast_done = false;        // the FP32 copies hold the coefficients of an execute
  bool owns_slot = true;         // false: fp32q reports into fp32's slot
  // the slot the plan's kernels report into (a refine plan's FP32 sweeps)
  int report_slot() const { return fp32 ? fp32->slot : slot; }
  ~Plan() {
    delete fp32q;
    delete fp32;
    if (ctx && owns_slot) status_slot_release(slot, ctx->device);
  }
};

// Memory of a plan: a job table (table_bytes) and scratch (scratch_bytes:
// each batched grid's region, then each alone-solved grid's buffer), every
// region 256-byte aligned; `offs` are relative to the scratch.  In one
// buffer the table comes first.  `order` gets the batched grids, heaviest
// lines first (tiles are dealt round-robin to the consumer warps, so this
// balances the tail).
template <typename F>
pentadStatus_t plan_layout(Context &ctx, int count, const pentadsolver_grid_t *grids,
                           int solvedim, std::vector<int> &order, std::vector<size_t> &offs,
                           std::vector<PlanSingle> &singles, bool &w2s, size_t &table_bytes,
                           size_t &scratch_bytes, const char **why,
                           std::vector<char> *grid_w2s = nullptr,
                           std::vector<char> *grid_loads = nullptr) {
  if (count < 1 || grids == nullptr) {
    *why = "no grids";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  const bool contig = solvedim == 0;
  std::vector<Shape> shapes(count);
  std::vector<char> ok(count, 0), need_w2s(count, 0), loads(count, 0);
  for (int i = 0; i < count; ++i) {
    const pentadsolver_grid_t &g = grids[i];
    pentadStatus_t st = make_shape(g.dims, g.ndim, solvedim, shapes[i], why);
    if (st != PENTAD_STATUS_SUCCESS) return st;
    if (!g.ds || !g.dl || !g.d || !g.du || !g.dw || !g.x) {
      *why = "an array pointer is null";
      return PENTAD_STATUS_INVALID_VALUE;
    }
    int w = 0;
    bool aligned = true;
    const void *ptrs[6] = {g.ds, g.dl, g.d, g.du, g.dw, g.x};
    for (const void *p : ptrs) aligned = aligned && reinterpret_cast<uintptr_t>(p) % sizeof(F) == 0;
    ok[i] = aligned && !env_flag("PENTA_NO_TMA") && tmem_shape<F>(shapes[i].L, contig, w);
    need_w2s[i] = (char)w;
    SolveArgs<F> ga{static_cast<const F *>(g.ds), static_cast<const F *>(g.dl),
                    static_cast<const F *>(g.d),  static_cast<const F *>(g.du),
                    static_cast<const F *>(g.dw), static_cast<F *>(g.x), shapes[i].L,
                    nullptr, 0, nullptr};
    loads[i] = (char)tmem_loads<F>(ga, contig);
  }
  (void)ctx;
  w2s = false;
  order.clear();
  for (int i = 0; i < count; ++i)
    if (ok[i]) {
      order.push_back(i);
      w2s = w2s || need_w2s[i] == 1 || need_w2s[i] == 2;  // factors through the buffer
    }
  // one job group per factor mode (du2 and dw2 in TMEM; du2 alone; all in
  // the buffer; all in TMEM) and stage layout (TMA tiles or bulk copies),
  // each heaviest lines first
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (need_w2s[a] != need_w2s[b]) return need_w2s[a] < need_w2s[b];
    if (loads[a] != loads[b]) return loads[a] < loads[b];
    return shapes[a].L.n > shapes[b].L.n;
  });
  table_bytes = round256(order.size() * tmem_job_bytes<F>());
  size_t off = 0;
  offs.assign(count, 0);
  for (int i : order) {
    offs[i] = off;
    off += round256(tmem_scratch_bytes<F>(shapes[i].L, contig, need_w2s[i]));
  }
  if (grid_w2s) *grid_w2s = need_w2s;
  if (grid_loads) *grid_loads = loads;
  singles.clear();
  for (int i = 0; i < count; ++i)
    if (!ok[i]) {
      const size_t b = buffer_bytes(shapes[i], sizeof(F));
      singles.push_back(PlanSingle{grids[i], off, b});
      off += round256(b);
    }
  scratch_bytes = off;
  return PENTAD_STATUS_SUCCESS;
}

template <typename F>
pentadStatus_t plan_build(Context &ctx, int count, const pentadsolver_grid_t *grids,
                          int solvedim, void *table_buf, size_t table_given, void *scratch_buf,
                          size_t scratch_given, int ctas, Plan *&out, const char **why) {
  if (!ctx.init()) {
    *why = "no usable CUDA device";
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  std::vector<int> order;
  std::vector<size_t> offs;
  std::vector<PlanSingle> singles;
  bool w2s = false;
  size_t table_bytes = 0, scratch_bytes = 0;
  std::vector<char> gw2s, gloads;
  pentadStatus_t st = plan_layout<F>(ctx, count, grids, solvedim, order, offs, singles, w2s,
                                     table_bytes, scratch_bytes, why, &gw2s, &gloads);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if ((table_bytes > 0 && (table_buf == nullptr || table_given < table_bytes ||
                           reinterpret_cast<uintptr_t>(table_buf) % 256 != 0)) ||
      (scratch_bytes > 0 && (scratch_buf == nullptr || scratch_given < scratch_bytes ||
                             reinterpret_cast<uintptr_t>(scratch_buf) % 256 != 0))) {
    *why = "the plan needs 256-byte aligned memory of the sizes pentadsolver_plan_buffer_size "
           "(or pentadsolver_plan_sizes) gives";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  unsigned char *base = static_cast<unsigned char *>(scratch_buf);
  unsigned char *table = static_cast<unsigned char *>(table_buf);
  std::vector<Plan::Group> groups;
  const bool contig = solvedim == 0;
  int total_tiles = 0;
  if (!order.empty()) {
    std::vector<SolveArgs<F>> args;
    std::vector<size_t> job_offs;
    for (int i : order) {
      const pentadsolver_grid_t &g = grids[i];
      Shape sh;
      make_shape(g.dims, g.ndim, solvedim, sh, why);
      args.push_back(SolveArgs<F>{static_cast<const F *>(g.ds), static_cast<const F *>(g.dl),
                                  static_cast<const F *>(g.d), static_cast<const F *>(g.du),
                                  static_cast<const F *>(g.dw), static_cast<F *>(g.x), sh.L,
                                  base + offs[i], 0, nullptr});
      job_offs.push_back(offs[i]);
    }
    const size_t jb = tmem_job_bytes<F>();
    void *host = std::aligned_alloc(64, round256(order.size() * jb));
    if (host == nullptr) {
      *why = "host memory for the job table";
      return PENTAD_STATUS_ALLOC_FAILED;
    }
    // fill each (factor mode, stage layout) group as its own tile list
    size_t first = 0;
    while (first < order.size()) {
      size_t last = first;
      while (last < order.size() && gw2s[order[last]] == gw2s[order[first]] &&
             gloads[order[last]] == gloads[order[first]])
        ++last;
      int tiles = 0;
      if (!tmem_fill_jobs<F>(args.data() + first, (int)(last - first), contig,
                             (int)gw2s[order[first]], (int)gloads[order[first]], base,
                             static_cast<unsigned char *>(host) + first * jb,
                             job_offs.data() + first, &tiles)) {
        std::free(host);
        *why = "tensor map encoding failed";
        return PENTAD_STATUS_INTERNAL_ERROR;
      }
      groups.push_back({(int)first, (int)(last - first), tiles, (int)gw2s[order[first]],
                        (int)gloads[order[first]]});
      total_tiles += tiles;
      first = last;
    }
    const cudaError_t e = copy_h2d(ctx, table, host, order.size() * jb);
    std::free(host);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *why = "copying the job table to the buffer";
      return PENTAD_STATUS_EXECUTION_FAILED;
    }
  }
  Plan *p = new Plan();
  p->ctx = &ctx;
  p->slot = status_slot_acquire();
  p->elem = sizeof(F);
  p->solvedim = solvedim;
  p->contig = contig;
  p->w2s = w2s;
  p->discard = true;  // every region is 256-byte aligned
  p->table = table;
  p->scratch = base;
  p->n_jobs = (int)order.size();
  p->total_tiles = total_tiles;
  p->groups = groups;
  {
    long long max_n = 0, lines = 0;
    for (int i : order) {
      Shape sh;
      make_shape(grids[i].dims, grids[i].ndim, solvedim, sh, why);
      max_n = std::max(max_n, sh.L.n);
      lines += sh.L.n_sys;
    }
    p->tkey = tune_key(ctx.gpu_name, "plan", sizeof(F), contig ? 0 : 1, max_n, lines);
  }
  if (ctas == 0) {  // the tuning table's CTA count for plans of this class
    TuneChoice tc;
    if (tune_lookup(p->tkey, tc) && tc.ctas > 0) ctas = tc.ctas;
  }
  p->ctas = (ctas > 0 && ctas < ctx.sm_count) ? ctas : ctx.sm_count;
  p->singles = singles;
  char d[160];
  int n_bulk = 0, n_x2t = 0;
  for (int i : order) {
    n_bulk += gloads[i] ? 1 : 0;
    n_x2t += gw2s[i] == 3 ? 1 : 0;
  }
  std::snprintf(d, sizeof d,
                "tmem-batch %s grids=%d tiles=%d launches=%d%s ctas=%d alone=%d pitched=%d "
                "x2t=%d",
                sizeof(F) == 8 ? "f64" : "f32", p->n_jobs, total_tiles, (int)groups.size(),
                w2s ? " w2s" : "", p->ctas, (int)singles.size(), n_bulk, n_x2t);
  p->desc = d;
  out = p;
  return PENTAD_STATUS_SUCCESS;
}

template <typename F> pentadStatus_t plan_run(Plan &p, cudaStream_t stream) {
  Context &ctx = *p.ctx;
  const char *why = "";
  if (!on_own_device(ctx, &why)) return PENTAD_STATUS_INVALID_VALUE;
  int *status = status_word(ctx.device, p.slot);
  if (status == nullptr) return PENTAD_STATUS_INTERNAL_ERROR;
  for (const Plan::Group &g : p.groups) {
    const cudaError_t e =
        launch_tmem_batch<F>(p.table + g.first * tmem_job_bytes<F>(), g.count, g.tiles,
                             p.contig, g.fmode, g.loads, p.discard, p.ctas, status, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return PENTAD_STATUS_EXECUTION_FAILED;
    }
  }
  for (const PlanSingle &s : p.singles) {
    const pentadStatus_t st =
        solve<F>(ctx, static_cast<const F *>(s.g.ds), static_cast<const F *>(s.g.dl),
                 static_cast<const F *>(s.g.d), static_cast<const F *>(s.g.du),
                 static_cast<const F *>(s.g.dw), static_cast<F *>(s.g.x), s.g.dims, s.g.ndim,
                 p.solvedim, p.scratch + s.offset, s.bytes, stream, &why, p.slot);
    if (st != PENTAD_STATUS_SUCCESS) return st;
  }
  return PENTAD_STATUS_SUCCESS;
}

// ---------------------------------------------------------------------------
// Mixed precision: FP32 sweeps, FP64 residual and correction
// ---------------------------------------------------------------------------
struct RefineLayout {
  size_t s_coef, r, b, solve, total;  // offsets (after a 256-byte estimate slot)
};
RefineLayout refine_layout(const Shape &sh) {
  const size_t N = (size_t)sh.L.n * (size_t)sh.L.n_sys;
  RefineLayout l;
  l.s_coef = 256;
  l.r = l.s_coef + round256(5 * N * sizeof(float));
  l.b = l.r + round256(N * sizeof(float));
  l.solve = l.b + round256(N * sizeof(double));
  l.total = l.solve + round256(buffer_bytes(sh, sizeof(float)));
  return l;
}

RefineGrid refine_grid(const Shape &sh, const double *ds, const double *dl, const double *d,
                       const double *du, const double *dw, double *x, unsigned char *coef32,
                       float *r, double *b, double *est) {
  const size_t N = (size_t)sh.L.n * (size_t)sh.L.n_sys;
  float *s = reinterpret_cast<float *>(coef32);
  RefineGrid g;
  std::memset(&g, 0, sizeof(g));
  g.ds = ds; g.dl = dl; g.d = d; g.du = du; g.dw = dw;
  g.x = x;
  g.b = b;
  g.s_ds = s; g.s_dl = s + N; g.s_d = s + 2 * N; g.s_du = s + 3 * N; g.s_dw = s + 4 * N;
  g.r = r;
  g.q = reinterpret_cast<float *>(b);  // one-step form: b is not copied, its slot holds q
  g.est = est;
  g.n_points = (long long)N;
  g.n = (int)sh.L.n;
  g.inner = (int)sh.L.inner;
  return g;
}

pentadStatus_t refine_solve(Context &ctx, const double *ds, const double *dl, const double *d,
                            const double *du, const double *dw, double *x, const int *dims,
                            int ndim, int solvedim, int steps, int reuse, void *buffer,
                            size_t bytes, cudaStream_t stream, const char **why) {
  Shape sh;
  pentadStatus_t st = make_shape(dims, ndim, solvedim, sh, why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (!ds || !dl || !d || !du || !dw || !x) {
    *why = "an array pointer is null";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (steps < 0 || steps > 8) {
    *why = "refinement steps must be in [0, 8]";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  const RefineLayout l = refine_layout(sh);
  if (buffer == nullptr || bytes < l.total || reinterpret_cast<uintptr_t>(buffer) % 256 != 0) {
    *why = "refinement needs a 256-byte aligned buffer of pentadsolver_refine_buffer_size bytes";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (!ctx.init()) {
    *why = "no usable CUDA device";
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  unsigned char *base = static_cast<unsigned char *>(buffer);
  const RefineGrid g = refine_grid(sh, ds, dl, d, du, dw, x, base + l.s_coef,
                                   reinterpret_cast<float *>(base + l.r),
                                   reinterpret_cast<double *>(base + l.b),
                                   reinterpret_cast<double *>(base));
  const int chunks = refine_chunks(g.n_points);
  auto step = [&](RefineStep k) {
    return launch_refine_step(k, g, nullptr, 1, chunks, stream) == cudaSuccess;
  };
  auto sweep = [&](float *rhs) {
    return solve<float>(ctx, g.s_ds, g.s_dl, g.s_d, g.s_du, g.s_dw, rhs, dims, ndim, solvedim,
                        base + l.solve, l.total - l.solve, stream, why);
  };
  if (steps <= 1) {  // the one-step form: no FP64 copies of x0 and b
    if (!step(reuse ? RefineStep::First : RefineStep::FirstCast)) goto failed;
    if ((st = sweep(g.r)) != PENTAD_STATUS_SUCCESS) return st;
    if (steps == 0) {
      if (!step(RefineStep::Lift)) goto failed;
      return PENTAD_STATUS_SUCCESS;
    }
    if (!step(RefineStep::Residual1)) goto failed;
    if ((st = sweep(g.q)) != PENTAD_STATUS_SUCCESS) return st;
    if (!step(RefineStep::Correct1)) goto failed;
    return PENTAD_STATUS_SUCCESS;
  }
  if (!step(reuse ? RefineStep::Prepare : RefineStep::PrepareCast)) goto failed;
  if ((st = sweep(g.r)) != PENTAD_STATUS_SUCCESS) return st;
  if (!step(RefineStep::Lift)) goto failed;
  for (int k = 0; k < steps; ++k) {
    if (!step(RefineStep::Residual)) goto failed;
    if ((st = sweep(g.r)) != PENTAD_STATUS_SUCCESS) return st;
    if (!step(RefineStep::Correct)) goto failed;
  }
  return PENTAD_STATUS_SUCCESS;
failed:
  cudaGetLastError();
  *why = "a refinement kernel failed to launch";
  return PENTAD_STATUS_EXECUTION_FAILED;
}

// Refine plans: [grid table][estimates][per grid: FP32 coefficients, r, b][FP32 plan]
pentadStatus_t refine_plan_layout(int count, const pentadsolver_grid_t *grids, int solvedim,
                                  std::vector<Shape> &shapes, std::vector<size_t> &goffs,
                                  size_t &fp32_off, const char **why) {
  if (count < 1 || grids == nullptr) {
    *why = "no grids";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  shapes.resize(count);
  goffs.resize(count);
  size_t off = round256(count * sizeof(RefineGrid)) + round256(count * 2 * sizeof(double));
  for (int i = 0; i < count; ++i) {
    pentadStatus_t st = make_shape(grids[i].dims, grids[i].ndim, solvedim, shapes[i], why);
    if (st != PENTAD_STATUS_SUCCESS) return st;
    const size_t N = (size_t)shapes[i].L.n * (size_t)shapes[i].L.n_sys;
    goffs[i] = off;
    off += round256(5 * N * sizeof(float)) + round256(N * sizeof(float)) +
           round256(N * sizeof(double));
  }
  fp32_off = off;
  return PENTAD_STATUS_SUCCESS;
}

// The FP32 grids of a refine plan (the cast coefficients and r, or with
// `on_q` the q array in the slot of b).
void refine_fp32_grids(int count, const pentadsolver_grid_t *grids,
                       const std::vector<Shape> &shapes, const std::vector<size_t> &goffs,
                       unsigned char *base, std::vector<pentadsolver_grid_t> &out,
                       bool on_q = false) {
  out.resize(count);
  for (int i = 0; i < count; ++i) {
    const size_t N = (size_t)shapes[i].L.n * (size_t)shapes[i].L.n_sys;
    float *s = reinterpret_cast<float *>(base + goffs[i]);
    float *r = reinterpret_cast<float *>(base + goffs[i] + round256(5 * N * sizeof(float)));
    out[i] = grids[i];
    out[i].ds = s; out[i].dl = s + N; out[i].d = s + 2 * N; out[i].du = s + 3 * N;
    out[i].dw = s + 4 * N;
    out[i].x = on_q ? reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(r) +
                                                round256(N * sizeof(float)))
                    : r;
  }
}

// ---------------------------------------------------------------------------
// Autotuning of single solves
// ---------------------------------------------------------------------------
struct TuneCandidate {
  const char *label, *spec, *algo;
  int lanes;
};
// Tensor-Memory kernel variants (forward ring and read-back stages), the older
// TMA kernels, the cp.async kernel with two lanes or one lane per line.
constexpr TuneCandidate kTuneCandidates[] = {
    {"tmem 2/4", "tmem=2,4", "thomas-pcr", 2}, {"tmem 2/3", "tmem=2,3", "thomas-pcr", 2},
    {"tmem 3/4", "tmem=3,4", "thomas-pcr", 2}, {"tmem 3/3", "tmem=3,3", "thomas-pcr", 2},
    {"tmem 3/2", "tmem=3,2", "thomas-pcr", 2}, {"tmem 4/3", "tmem=4,3", "thomas-pcr", 2},
    {"tma", "no-tmem", "thomas-pcr", 2},       {"cp.async P2", "no-tma", "thomas-pcr", 2},
    {"cp.async P1", "no-tma", "thomas-pcr", 1},
};

// Times every candidate on the caller's problem (x is overwritten by the
// trials; x_save, when given, keeps and restores it), records the fastest in
// the tuning table and writes a report: one line per distinct kernel variant,
// "label\tspec\talgo\tlanes\tvariant\tms", the fastest first.
template <typename F>
pentadStatus_t autotune_solve(Context &ctx, const F *ds, const F *dl, const F *d, const F *du,
                              const F *dw, F *x, F *x_save, const int *dims, int ndim,
                              int solvedim, void *buf, size_t buf_bytes, int reps,
                              cudaStream_t stream, std::string &report, const char **why) {
  Shape sh;
  pentadStatus_t st = make_shape(dims, ndim, solvedim, sh, why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (reps < 1 || reps > 1000) {
    *why = "reps out of range";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (!ctx.init()) {
    *why = "no usable CUDA device";
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  if (!on_own_device(ctx, why)) return PENTAD_STATUS_INVALID_VALUE;
  const size_t bytes = (size_t)sh.L.n * (size_t)sh.L.n_sys * sizeof(F);
  if (x_save != nullptr &&
      cudaMemcpyAsync(x_save, x, bytes, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  const int dir = sh.dir;
  struct Row {
    const TuneCandidate *c;
    std::string variant;
    float ms;
  };
  std::vector<Row> rows;
  std::unordered_set<std::string> seen;
  pentadStatus_t out = PENTAD_STATUS_SUCCESS;
  for (const TuneCandidate &c : kTuneCandidates) {
    Context trial;
    trial.init();
    trial.slot = ctx.slot;
    trial.tuning[dir] = c.spec;
    trial.forced[dir] = parse_algo(c.algo);
    trial.forced_lanes[dir] = c.lanes;
    const char *w = "";
    if (solve<F>(trial, ds, dl, d, du, dw, x, dims, ndim, solvedim, buf, buf_bytes, stream,
                 &w) != PENTAD_STATUS_SUCCESS) {
      cudaGetLastError();
      continue;
    }
    const std::string variant = trial.variant[dir];
    if (!seen.insert(variant).second) continue;  // the shape sent it to a kernel timed already
    bool ok = cudaEventRecord(e0, stream) == cudaSuccess;
    for (int r = 0; ok && r < reps; ++r)
      ok = solve<F>(trial, ds, dl, d, du, dw, x, dims, ndim, solvedim, buf, buf_bytes, stream,
                    &w) == PENTAD_STATUS_SUCCESS;
    float ms = 0.f;
    ok = ok && cudaEventRecord(e1, stream) == cudaSuccess &&
         cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      out = PENTAD_STATUS_EXECUTION_FAILED;
      break;
    }
    rows.push_back(Row{&c, variant, ms / reps});
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (x_save != nullptr &&
      cudaMemcpyAsync(x, x_save, bytes, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) {
    cudaGetLastError();
    out = PENTAD_STATUS_EXECUTION_FAILED;
  }
  if (out != PENTAD_STATUS_SUCCESS) return out;
  if (rows.empty()) {
    *why = "no candidate ran";
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  std::stable_sort(rows.begin(), rows.end(), [](const Row &a, const Row &b) { return a.ms < b.ms; });
  TuneChoice best;
  best.spec = rows[0].c->spec;
  best.algo = rows[0].c->algo;
  best.lanes = rows[0].c->lanes;
  best.ms = rows[0].ms;
  tune_store(tune_key(ctx.gpu_name, "solve", sizeof(F), dir, sh.L.n, sh.L.n_sys), best);
  report.clear();
  for (const Row &r : rows) {
    char ms[32];
    std::snprintf(ms, sizeof ms, "%.6g", r.ms);
    report += std::string(r.c->label) + "\t" + r.c->spec + "\t" + r.c->algo + "\t" +
              std::to_string(r.c->lanes) + "\t" + r.variant + "\t" + ms + "\n";
  }
  return PENTAD_STATUS_SUCCESS;
}

bool copy_out(const std::string &v, char *out, size_t len) {
  if (out == nullptr || len == 0) return out == nullptr;
  if (v.size() + 1 > len) return false;
  std::memcpy(out, v.c_str(), v.size() + 1);
  return true;
}

// Read and clear one status slot; ZERO_PIVOT when bit 0 was set.
pentadStatus_t take_status(int device, int slot, cudaStream_t stream, int *bits) {
  int host = 0;
  if (status_take(device, slot, stream, &host) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  if (bits) *bits = host;
  return (host & STATUS_ZERO_PIVOT_BIT) ? PENTAD_STATUS_ZERO_PIVOT : PENTAD_STATUS_SUCCESS;
}

size_t size_query(const int *dims, int ndim, int solvedim, size_t elem) {
  Shape sh;
  const char *why = "";
  if (make_shape(dims, ndim, solvedim, sh, &why) != PENTAD_STATUS_SUCCESS)
    return 0;
  return buffer_bytes(sh, elem);
}

}  // namespace

pentadStatus_t check_shape(const int *dims, int ndim, int solvedim, Lines &L, const char **why) {
  Shape sh;
  const pentadStatus_t st = make_shape(dims, ndim, solvedim, sh, why);
  if (st == PENTAD_STATUS_SUCCESS) L = sh.L;
  return st;
}

pentadStatus_t bind_handle(pentadsolver_handle_t h, int **status, const char **why) {
  Context *ctx = resolve(h);
  if (!ctx->init()) {
    *why = "no usable CUDA device";
    return PENTAD_STATUS_NOT_INITIALIZED;
  }
  if (!on_own_device(*ctx, why)) return PENTAD_STATUS_INVALID_VALUE;
  *status = status_word(ctx->device, ctx->slot);
  if (*status == nullptr) {
    *why = "cannot address the device status word";
    return PENTAD_STATUS_INTERNAL_ERROR;
  }
  return PENTAD_STATUS_SUCCESS;
}

}  // namespace penta

using penta::Context;

// ===========================================================================
// Reference-named C ABI (include/pentadsolver.hpp)
// ===========================================================================
extern "C" void pentadsolver_create(pentadsolver_handle_t *handle,
                                    void * /*communicator*/, int /*ndims*/,
                                    const int * /*num_procs*/) {
  if (handle == nullptr) return;
  auto *c = new Context();
  c->slot = penta::status_slot_acquire();
  {
    std::lock_guard<std::mutex> lock(penta::g_reg_mu);
    penta::g_live.insert(c);
  }
  *handle = c;
}

extern "C" void pentadsolver_destroy(pentadsolver_handle_t *handle) {
  if (handle == nullptr || *handle == nullptr) return;
  auto *c = static_cast<Context *>(*handle);
  bool owned = false;
  {
    std::lock_guard<std::mutex> lock(penta::g_reg_mu);
    owned = penta::g_live.erase(c) > 0;
  }
  if (owned) {
    penta::status_slot_release(c->slot, c->device);
    delete c;
  }
  *handle = nullptr;
}

extern "C" size_t pentadsolver_D_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t, const double *, const double *, const double *,
    const double *, const double *, const double *, const int *t_dims,
    int t_ndim, int t_solvedim) {
  return penta::size_query(t_dims, t_ndim, t_solvedim, sizeof(double));
}
extern "C" size_t pentadsolver_S_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t, const float *, const float *, const float *,
    const float *, const float *, const float *, const int *t_dims,
    int t_ndim, int t_solvedim) {
  return penta::size_query(t_dims, t_ndim, t_solvedim, sizeof(float));
}
size_t pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t h, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, const double *x,
    const int *t_dims, int t_ndim, int t_solvedim) {
  return pentadsolver_D_gpsv_batch_buffer_size_ext(h, ds, dl, d, du, dw, x,
                                                   t_dims, t_ndim, t_solvedim);
}
size_t pentadsolver_gpsv_batch_buffer_size_ext(
    pentadsolver_handle_t h, const float *ds, const float *dl, const float *d,
    const float *du, const float *dw, const float *x, const int *t_dims,
    int t_ndim, int t_solvedim) {
  return pentadsolver_S_gpsv_batch_buffer_size_ext(h, ds, dl, d, du, dw, x,
                                                   t_dims, t_ndim, t_solvedim);
}

extern "C" void pentadsolver_D_gpsv_batch(pentadsolver_handle_t h,
                                          const double *ds, const double *dl,
                                          const double *d, const double *du,
                                          const double *dw, double *x,
                                          const int *t_dims, int t_ndim,
                                          int t_solvedim, void *t_buffer) {
  penta::solve_void<double>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                            t_solvedim, t_buffer);
}
extern "C" void pentadsolver_S_gpsv_batch(pentadsolver_handle_t h,
                                          const float *ds, const float *dl,
                                          const float *d, const float *du,
                                          const float *dw, float *x,
                                          const int *t_dims, int t_ndim,
                                          int t_solvedim, void *t_buffer) {
  penta::solve_void<float>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                           t_solvedim, t_buffer);
}
void pentadsolver_gpsv_batch(pentadsolver_handle_t h, const double *ds,
                             const double *dl, const double *d,
                             const double *du, const double *dw, double *x,
                             const int *t_dims, int t_ndim, int t_solvedim,
                             void *t_buffer) {
  penta::solve_void<double>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                            t_solvedim, t_buffer);
}
void pentadsolver_gpsv_batch(pentadsolver_handle_t h, const float *ds,
                             const float *dl, const float *d, const float *du,
                             const float *dw, float *x, const int *t_dims,
                             int t_ndim, int t_solvedim, void *t_buffer) {
  penta::solve_void<float>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                           t_solvedim, t_buffer);
}

extern "C" const char *pentadsolver_kernel_that_ran(int dir) {
  return (dir >= 0 && dir < 3) ? penta::g_ran[dir].load() : penta::kNone;
}

// ===========================================================================
// Two-buffer form (include/pentadsolver_cuda.hpp; that header shares its
// include guard with pentadsolver.hpp, so the exports are marked here)
// ===========================================================================
extern "C" PENTAD_API void pentadsolver_D_gpsv_batch_buffer_size_two_buffer(
    pentadsolver_handle_t, const double *, const double *, const double *,
    const double *, const double *, const double *, const int *t_dims,
    int t_ndim, int t_solvedim, size_t *host_bytes, size_t *device_bytes) {
  if (host_bytes) *host_bytes = 0;
  if (device_bytes)
    *device_bytes = penta::size_query(t_dims, t_ndim, t_solvedim, sizeof(double));
}
extern "C" PENTAD_API void pentadsolver_S_gpsv_batch_buffer_size_two_buffer(
    pentadsolver_handle_t, const float *, const float *, const float *,
    const float *, const float *, const float *, const int *t_dims,
    int t_ndim, int t_solvedim, size_t *host_bytes, size_t *device_bytes) {
  if (host_bytes) *host_bytes = 0;
  if (device_bytes)
    *device_bytes = penta::size_query(t_dims, t_ndim, t_solvedim, sizeof(float));
}
extern "C" PENTAD_API void pentadsolver_D_gpsv_batch_two_buffer(
    pentadsolver_handle_t h, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void * /*t_buffer_h*/,
    void *t_buffer_d) {
  penta::solve_void<double>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                            t_solvedim, t_buffer_d);
}
extern "C" PENTAD_API void pentadsolver_S_gpsv_batch_two_buffer(
    pentadsolver_handle_t h, const float *ds, const float *dl, const float *d,
    const float *du, const float *dw, float *x, const int *t_dims, int t_ndim,
    int t_solvedim, void * /*t_buffer_h*/, void *t_buffer_d) {
  penta::solve_void<float>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                           t_solvedim, t_buffer_d);
}

// ===========================================================================
// Extension C ABI (include/pentadsolver_ext.h)
// ===========================================================================
extern "C" pentadStatus_t pentadsolver_buffer_size_ex(
    pentadsolver_handle_t, int elem_bytes, const int *t_dims, int t_ndim,
    int t_solvedim, size_t *bytes) {
  if (bytes == nullptr || (elem_bytes != 4 && elem_bytes != 8))
    return PENTAD_STATUS_INVALID_VALUE;
  penta::Shape sh;
  const char *why = "";
  pentadStatus_t st = penta::make_shape(t_dims, t_ndim, t_solvedim, sh, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  *bytes = penta::buffer_bytes(sh, (size_t)elem_bytes);
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_D_gpsv_batch_ex(
    pentadsolver_handle_t h, const double *ds, const double *dl,
    const double *d, const double *du, const double *dw, double *x,
    const int *t_dims, int t_ndim, int t_solvedim, void *t_buffer,
    size_t t_buffer_bytes, void *stream) {
  return penta::solve_ex<double>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                                 t_solvedim, t_buffer, t_buffer_bytes, stream);
}
extern "C" pentadStatus_t pentadsolver_S_gpsv_batch_ex(
    pentadsolver_handle_t h, const float *ds, const float *dl, const float *d,
    const float *du, const float *dw, float *x, const int *t_dims, int t_ndim,
    int t_solvedim, void *t_buffer, size_t t_buffer_bytes, void *stream) {
  return penta::solve_ex<float>(h, ds, dl, d, du, dw, x, t_dims, t_ndim,
                                t_solvedim, t_buffer, t_buffer_bytes, stream);
}

extern "C" pentadStatus_t pentadsolver_status_check(pentadsolver_handle_t h,
                                                    void *stream, int *bits) {
  Context *ctx = penta::resolve(h);
  if (!ctx->init()) return PENTAD_STATUS_NOT_INITIALIZED;
  const char *why = "";
  if (!penta::on_own_device(*ctx, &why)) return PENTAD_STATUS_INVALID_VALUE;
  return penta::take_status(ctx->device, ctx->slot, static_cast<cudaStream_t>(stream), bits);
}

extern "C" pentadStatus_t pentadsolver_selftest_bounded_wait(pentadsolver_handle_t h,
                                                             unsigned limit_us, void *stream) {
  if (limit_us == 0 || limit_us > 1000000u) return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  if (!ctx->init()) return PENTAD_STATUS_NOT_INITIALIZED;
  const char *why = "";
  if (!penta::on_own_device(*ctx, &why)) return PENTAD_STATUS_INVALID_VALUE;
  int *word = penta::status_word(ctx->device, ctx->slot);
  if (word == nullptr) return PENTAD_STATUS_INTERNAL_ERROR;
  if (penta::launch_bounded_wait_selftest(1000ull * limit_us, word,
                                          static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_set_algo(pentadsolver_handle_t h,
                                                int dir, const char *algo,
                                                int pcr_lanes) {
  if (dir < 0 || dir > 2) return PENTAD_STATUS_INVALID_VALUE;
  penta::Algo a = penta::parse_algo(algo);
  if (a == penta::Algo::Unknown) return PENTAD_STATUS_INVALID_VALUE;
  if (pcr_lanes != 0 && pcr_lanes != 1 && pcr_lanes != 2 && pcr_lanes != 4 &&
      pcr_lanes != 8 && pcr_lanes != 16 && pcr_lanes != 32)
    return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->forced[dir] = a;
  ctx->forced_lanes[dir] = pcr_lanes;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_set_tuning(pentadsolver_handle_t h, int dir,
                                                  const char *spec) {
  if (dir < 0 || dir > 2) return PENTAD_STATUS_INVALID_VALUE;
  std::string v = spec ? spec : "";
  if (v == "auto") v.clear();
  const bool ok = v.empty() || v == "no-tma" || v == "no-tmem" || v.rfind("tmem=", 0) == 0 ||
                  v.rfind("tma=", 0) == 0;
  if (!ok) return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->tuning[dir] = v;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" const char *pentadsolver_kernel_that_ran_ex(pentadsolver_handle_t h,
                                                       int dir) {
  if (dir < 0 || dir > 2) return penta::kNone;
  return penta::resolve(h)->ran[dir].load();
}

extern "C" const char *pentadsolver_variant_that_ran(pentadsolver_handle_t h,
                                                     int dir) {
  if (dir < 0 || dir > 2) return penta::kNone;
  Context *ctx = penta::resolve(h);
  thread_local std::string out;
  std::lock_guard<std::mutex> lock(ctx->mu);
  out = ctx->variant[dir].empty() ? std::string(penta::kNone) : ctx->variant[dir];
  return out.c_str();
}

extern "C" const char *pentadsolver_status_string(pentadStatus_t s) {
  switch (s) {
    case PENTAD_STATUS_SUCCESS: return "success";
    case PENTAD_STATUS_NOT_INITIALIZED: return "not initialized";
    case PENTAD_STATUS_ALLOC_FAILED: return "allocation failed";
    case PENTAD_STATUS_INVALID_VALUE: return "invalid value";
    case PENTAD_STATUS_ARCH_MISMATCH: return "architecture mismatch";
    case PENTAD_STATUS_MAPPING_ERROR: return "mapping error";
    case PENTAD_STATUS_EXECUTION_FAILED: return "execution failed";
    case PENTAD_STATUS_INTERNAL_ERROR: return "internal error";
    case PENTAD_STATUS_MATRIX_TYPE_NOT_SUPPORTED: return "matrix type not supported";
    case PENTAD_STATUS_ZERO_PIVOT: return "zero pivot";
  }
  return "unknown status";
}

// ===========================================================================
// Plans and mixed-precision refinement (pentadsolver_ext.h)
// ===========================================================================
struct pentadsolver_plan_s {
  penta::Plan *p;
};

extern "C" pentadStatus_t pentadsolver_plan_status_check(pentadsolver_plan_t plan, void *stream,
                                                         int *bits) {
  if (plan == nullptr || plan->p == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  const penta::Plan &p = *plan->p;
  const char *why = "";
  if (!penta::on_own_device(*p.ctx, &why)) return PENTAD_STATUS_INVALID_VALUE;
  return penta::take_status(p.ctx->device, p.report_slot(), static_cast<cudaStream_t>(stream),
                            bits);
}

extern "C" pentadStatus_t pentadsolver_plan_buffer_size(pentadsolver_handle_t h, int elem_bytes,
                                                        int count,
                                                        const pentadsolver_grid_t *grids,
                                                        int solvedim, size_t *bytes) {
  if (bytes == nullptr || (elem_bytes != 4 && elem_bytes != 8)) return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  std::vector<int> order;
  std::vector<size_t> offs;
  std::vector<penta::PlanSingle> singles;
  bool w2s = false;
  const char *why = "";
  size_t tb = 0, sb = 0;
  pentadStatus_t st =
      elem_bytes == 8
          ? penta::plan_layout<double>(*ctx, count, grids, solvedim, order, offs, singles, w2s,
                                       tb, sb, &why)
          : penta::plan_layout<float>(*ctx, count, grids, solvedim, order, offs, singles, w2s,
                                      tb, sb, &why);
  *bytes = tb + sb;
  return st;
}

extern "C" pentadStatus_t pentadsolver_plan_sizes(pentadsolver_handle_t h, int elem_bytes,
                                                  int count, const pentadsolver_grid_t *grids,
                                                  int solvedim, size_t *table_bytes,
                                                  size_t *scratch_bytes) {
  if (table_bytes == nullptr || scratch_bytes == nullptr || (elem_bytes != 4 && elem_bytes != 8))
    return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  std::vector<int> order;
  std::vector<size_t> offs;
  std::vector<penta::PlanSingle> singles;
  bool w2s = false;
  const char *why = "";
  return elem_bytes == 8
             ? penta::plan_layout<double>(*ctx, count, grids, solvedim, order, offs, singles,
                                          w2s, *table_bytes, *scratch_bytes, &why)
             : penta::plan_layout<float>(*ctx, count, grids, solvedim, order, offs, singles, w2s,
                                         *table_bytes, *scratch_bytes, &why);
}

extern "C" pentadStatus_t pentadsolver_plan_create(pentadsolver_handle_t h, int elem_bytes,
                                                   int count, const pentadsolver_grid_t *grids,
                                                   int solvedim, void *buffer,
                                                   size_t buffer_bytes, int ctas,
                                                   pentadsolver_plan_t *plan) {
  if (plan == nullptr || (elem_bytes != 4 && elem_bytes != 8)) return PENTAD_STATUS_INVALID_VALUE;
  *plan = nullptr;
  size_t tb = 0, sb = 0;
  pentadStatus_t st = pentadsolver_plan_sizes(h, elem_bytes, count, grids, solvedim, &tb, &sb);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (buffer == nullptr || buffer_bytes < tb + sb) return PENTAD_STATUS_INVALID_VALUE;
  unsigned char *b = static_cast<unsigned char *>(buffer);
  return pentadsolver_plan_create_split(h, elem_bytes, count, grids, solvedim, b, tb, b + tb,
                                        buffer_bytes - tb, ctas, plan);
}

extern "C" pentadStatus_t pentadsolver_plan_create_split(
    pentadsolver_handle_t h, int elem_bytes, int count, const pentadsolver_grid_t *grids,
    int solvedim, void *table, size_t table_bytes, void *scratch, size_t scratch_bytes, int ctas,
    pentadsolver_plan_t *plan) {
  if (plan == nullptr || (elem_bytes != 4 && elem_bytes != 8)) return PENTAD_STATUS_INVALID_VALUE;
  *plan = nullptr;
  Context *ctx = penta::resolve(h);
  penta::Plan *p = nullptr;
  const char *why = "";
  pentadStatus_t st =
      elem_bytes == 8
          ? penta::plan_build<double>(*ctx, count, grids, solvedim, table, table_bytes, scratch,
                                      scratch_bytes, ctas, p, &why)
          : penta::plan_build<float>(*ctx, count, grids, solvedim, table, table_bytes, scratch,
                                     scratch_bytes, ctas, p, &why);
  if (st != PENTAD_STATUS_SUCCESS) {
    if (penta::env_flag("PENTA_DEBUG_LAUNCH")) std::fprintf(stderr, "[penta] plan: %s\n", why);
    return st;
  }
  *plan = new pentadsolver_plan_s{p};
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_plan_execute_ex(pentadsolver_plan_t plan, void *stream,
                                                     int flags) {
  if (plan == nullptr || plan->p == nullptr || (flags & ~PENTADSOLVER_PLAN_REUSE_FP32) != 0)
    return PENTAD_STATUS_INVALID_VALUE;
  penta::Plan &p = *plan->p;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!p.refine)
    return p.elem == 8 ? penta::plan_run<double>(p, s) : penta::plan_run<float>(p, s);
  // refinement: cast, FP32 sweep, lift, then (residual, sweep, correct) x steps
  auto step = [&](penta::RefineStep k) {
    penta::RefineGrid none;
    std::memset(&none, 0, sizeof(none));
    return penta::launch_refine_step(k, none, p.rtable, p.count, p.chunks, s) == cudaSuccess;
  };
  pentadStatus_t st;
  // the FP32 copies are cast again unless the caller vouches that the
  // coefficients did not change since an execute that cast them
  const bool cast = !(p.cast_done && (flags & PENTADSOLVER_PLAN_REUSE_FP32));
  p.cast_done = false;  // set again once this execute's cast is queued
  if (p.steps <= 1) {  // the one-step form: no FP64 copies of x0 and b
    if (!step(cast ? penta::RefineStep::FirstCast : penta::RefineStep::First))
      return PENTAD_STATUS_EXECUTION_FAILED;
    p.cast_done = true;
    if ((st = penta::plan_run<float>(*p.fp32, s)) != PENTAD_STATUS_SUCCESS) return st;
    if (p.steps == 0)
      return step(penta::RefineStep::Lift) ? PENTAD_STATUS_SUCCESS
                                           : PENTAD_STATUS_EXECUTION_FAILED;
    if (!step(penta::RefineStep::Residual1)) return PENTAD_STATUS_EXECUTION_FAILED;
    if ((st = penta::plan_run<float>(*p.fp32q, s)) != PENTAD_STATUS_SUCCESS) return st;
    return step(penta::RefineStep::Correct1) ? PENTAD_STATUS_SUCCESS
                                             : PENTAD_STATUS_EXECUTION_FAILED;
  }
  if (!step(cast ? penta::RefineStep::PrepareCast : penta::RefineStep::Prepare))
    return PENTAD_STATUS_EXECUTION_FAILED;
  p.cast_done = true;
  if ((st = penta::plan_run<float>(*p.fp32, s)) != PENTAD_STATUS_SUCCESS) return st;
  if (!step(penta::RefineStep::Lift)) return PENTAD_STATUS_EXECUTION_FAILED;
  for (int k = 0; k < p.steps; ++k) {
    if (!step(penta::RefineStep::Residual)) return PENTAD_STATUS_EXECUTION_FAILED;
    if ((st = penta::plan_run<float>(*p.fp32, s)) != PENTAD_STATUS_SUCCESS) return st;
    if (!step(penta::RefineStep::Correct)) return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_plan_execute(pentadsolver_plan_t plan, void *stream) {
  return pentadsolver_plan_execute_ex(plan, stream, 0);
}

extern "C" const char *pentadsolver_plan_describe(pentadsolver_plan_t plan) {
  if (plan == nullptr || plan->p == nullptr) return penta::kNone;
  return plan->p->desc.c_str();
}

extern "C" pentadStatus_t pentadsolver_plan_destroy(pentadsolver_plan_t plan) {
  if (plan == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  delete plan->p;
  delete plan;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_refine_buffer_size(pentadsolver_handle_t, const int *dims,
                                                          int ndim, int solvedim,
                                                          size_t *bytes) {
  if (bytes == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  penta::Shape sh;
  const char *why = "";
  pentadStatus_t st = penta::make_shape(dims, ndim, solvedim, sh, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  *bytes = penta::refine_layout(sh).total;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_D_gpsv_batch_refine(
    pentadsolver_handle_t h, const double *ds, const double *dl, const double *d,
    const double *du, const double *dw, double *x, const int *dims, int ndim, int solvedim,
    int steps, int reuse_fp32_coefficients, void *buffer, size_t buffer_bytes, void *stream) {
  Context *ctx = penta::resolve(h);
  const char *why = "";
  pentadStatus_t st = penta::refine_solve(*ctx, ds, dl, d, du, dw, x, dims, ndim, solvedim,
                                          steps, reuse_fp32_coefficients, buffer, buffer_bytes,
                                          static_cast<cudaStream_t>(stream), &why);
  if (st != PENTAD_STATUS_SUCCESS && penta::env_flag("PENTA_DEBUG_LAUNCH"))
    std::fprintf(stderr, "[penta] refine: %s\n", why);
  return st;
}

extern "C" pentadStatus_t pentadsolver_refine_estimate(const void *buffer, void *stream,
                                                       double *out) {
  if (buffer == nullptr || out == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(out, buffer, 2 * sizeof(double), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_refine_plan_buffer_size(pentadsolver_handle_t h,
                                                               int count,
                                                               const pentadsolver_grid_t *grids,
                                                               int solvedim, size_t *bytes) {
  if (bytes == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  std::vector<penta::Shape> shapes;
  std::vector<size_t> goffs;
  size_t fp32_off = 0;
  const char *why = "";
  pentadStatus_t st =
      penta::refine_plan_layout(count, grids, solvedim, shapes, goffs, fp32_off, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  // the FP32 plan's own layout over the cast grids (pointers do not matter here)
  std::vector<pentadsolver_grid_t> g32;
  penta::refine_fp32_grids(count, grids, shapes, goffs,
                           reinterpret_cast<unsigned char *>(uintptr_t(256)), g32);
  // two job tables (over r, and over q for the one-step form), one scratch
  size_t tb = 0, sb = 0;
  st = pentadsolver_plan_sizes(h, 4, count, g32.data(), solvedim, &tb, &sb);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  *bytes = fp32_off + 2 * penta::round256(tb) + sb;
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_refine_plan_create(pentadsolver_handle_t h, int count,
                                                          const pentadsolver_grid_t *grids,
                                                          int solvedim, int steps, void *buffer,
                                                          size_t buffer_bytes, int ctas,
                                                          pentadsolver_plan_t *plan) {
  if (plan == nullptr || steps < 0 || steps > 8) return PENTAD_STATUS_INVALID_VALUE;
  *plan = nullptr;
  size_t need = 0;
  pentadStatus_t st = pentadsolver_refine_plan_buffer_size(h, count, grids, solvedim, &need);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  if (buffer == nullptr || buffer_bytes < need || reinterpret_cast<uintptr_t>(buffer) % 256 != 0)
    return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  if (!ctx->init()) return PENTAD_STATUS_NOT_INITIALIZED;
  std::vector<penta::Shape> shapes;
  std::vector<size_t> goffs;
  size_t fp32_off = 0;
  const char *why = "";
  st = penta::refine_plan_layout(count, grids, solvedim, shapes, goffs, fp32_off, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  unsigned char *base = static_cast<unsigned char *>(buffer);
  std::vector<pentadsolver_grid_t> g32;
  penta::refine_fp32_grids(count, grids, shapes, goffs, base, g32);
  penta::Plan *fp32 = nullptr;
  size_t tb = 0, sb = 0;
  st = pentadsolver_plan_sizes(h, 4, count, g32.data(), solvedim, &tb, &sb);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  std::string rkey;
  {
    long long max_n = 0, lines = 0;
    for (const penta::Shape &sh : shapes) {
      max_n = std::max(max_n, sh.L.n);
      lines += sh.L.n_sys;
    }
    rkey = penta::tune_key(ctx->gpu_name, "refine", 8, solvedim == 0 ? 0 : 1, max_n, lines);
    penta::TuneChoice tc;
    if (ctas == 0 && penta::tune_lookup(rkey, tc) && tc.ctas > 0) ctas = tc.ctas;
  }
  const size_t tb2 = 2 * penta::round256(tb);
  st = penta::plan_build<float>(*ctx, count, g32.data(), solvedim, base + fp32_off, tb,
                                base + fp32_off + tb2, buffer_bytes - fp32_off - tb2, ctas, fp32,
                                &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  penta::Plan *fp32q = nullptr;
  if (steps == 1) {  // the second sweep of the one-step form solves q in place
    std::vector<pentadsolver_grid_t> g32q;
    penta::refine_fp32_grids(count, grids, shapes, goffs, base, g32q, true);
    st = penta::plan_build<float>(*ctx, count, g32q.data(), solvedim,
                                  base + fp32_off + penta::round256(tb), tb, base + fp32_off + tb2,
                                  buffer_bytes - fp32_off - tb2, ctas, fp32q, &why);
    if (st != PENTAD_STATUS_SUCCESS) {
      delete fp32;
      return st;
    }
    penta::status_slot_release(fp32q->slot, ctx->device);  // report with the first sweep
    fp32q->slot = fp32->slot;
    fp32q->owns_slot = false;
  }
  // the grid table of the FP64 steps
  std::vector<penta::RefineGrid> table(count);
  double *est = reinterpret_cast<double *>(base + penta::round256(count * sizeof(penta::RefineGrid)));
  int chunks = 0;
  for (int i = 0; i < count; ++i) {
    const pentadsolver_grid_t &g = grids[i];
    const size_t N = (size_t)shapes[i].L.n * (size_t)shapes[i].L.n_sys;
    unsigned char *gb = base + goffs[i];
    float *r = reinterpret_cast<float *>(gb + penta::round256(5 * N * sizeof(float)));
    double *b = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(r) +
                                           penta::round256(N * sizeof(float)));
    table[i] = penta::refine_grid(shapes[i], static_cast<const double *>(g.ds),
                                  static_cast<const double *>(g.dl),
                                  static_cast<const double *>(g.d),
                                  static_cast<const double *>(g.du),
                                  static_cast<const double *>(g.dw), static_cast<double *>(g.x),
                                  gb, r, b, est + 2 * i);
    table[i].chunk_base = chunks;
    chunks += penta::refine_chunks(table[i].n_points);
  }
  if (penta::copy_h2d(*ctx, base, table.data(), count * sizeof(penta::RefineGrid)) !=
      cudaSuccess) {
    cudaGetLastError();
    delete fp32q;
    delete fp32;
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  penta::Plan *p = new penta::Plan();
  p->ctx = ctx;
  p->elem = 8;
  p->solvedim = solvedim;
  p->refine = true;
  p->steps = steps;
  p->chunks = chunks;
  p->rtable = reinterpret_cast<penta::RefineGrid *>(base);
  p->est = est;
  p->count = count;
  p->fp32 = fp32;
  p->fp32q = fp32q;
  p->tkey = rkey;
  p->desc = "refine steps=" + std::to_string(steps) + " over " + fp32->desc;
  *plan = new pentadsolver_plan_s{p};
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_plan_estimates(pentadsolver_plan_t plan, void *stream,
                                                      double *out) {
  if (plan == nullptr || plan->p == nullptr || !plan->p->refine || out == nullptr)
    return PENTAD_STATUS_INVALID_VALUE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(out, plan->p->est, 2 * plan->p->count * sizeof(double),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

// ===========================================================================
// Tuning table and autotuning (pentadsolver_ext.h)
// ===========================================================================
extern "C" pentadStatus_t pentadsolver_tuning_load(const char *path) {
  if (path == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  return penta::tune_load(path) ? PENTAD_STATUS_SUCCESS : PENTAD_STATUS_INVALID_VALUE;
}

extern "C" pentadStatus_t pentadsolver_tuning_save(const char *path) {
  if (path == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  return penta::tune_save(path) ? PENTAD_STATUS_SUCCESS : PENTAD_STATUS_INVALID_VALUE;
}

extern "C" pentadStatus_t pentadsolver_tuning_clear(void) {
  penta::tune_clear();
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_tuning_set(const char *key, const char *spec,
                                                  const char *algo, int lanes, int ctas,
                                                  double ms) {
  if (key == nullptr || key[0] == '\0' || lanes < 0 || lanes > 32 || ctas < 0)
    return PENTAD_STATUS_INVALID_VALUE;
  std::string sp = spec ? spec : "";
  if (sp == "auto") sp.clear();
  if (!(sp.empty() || sp == "no-tma" || sp == "no-tmem" || sp.rfind("tmem=", 0) == 0 ||
        sp.rfind("tma=", 0) == 0))
    return PENTAD_STATUS_INVALID_VALUE;
  std::string al = algo ? algo : "";
  if (al == "auto") al.clear();
  if (!al.empty() && penta::parse_algo(al.c_str()) == penta::Algo::Unknown)
    return PENTAD_STATUS_INVALID_VALUE;
  penta::TuneChoice c;
  c.spec = sp;
  c.algo = al;
  c.lanes = lanes;
  c.ctas = ctas;
  c.ms = ms;
  penta::tune_store(key, c);
  return PENTAD_STATUS_SUCCESS;
}

extern "C" pentadStatus_t pentadsolver_tuning_lookup(const char *key, char *out, size_t len) {
  if (key == nullptr) return PENTAD_STATUS_INVALID_VALUE;
  penta::TuneChoice c;
  if (!penta::tune_lookup(key, c)) return PENTAD_STATUS_INVALID_VALUE;
  return penta::copy_out(penta::tune_format(c), out, len) ? PENTAD_STATUS_SUCCESS
                                                          : PENTAD_STATUS_INVALID_VALUE;
}

extern "C" pentadStatus_t pentadsolver_tuning_key(const char *gpu_name, const char *kind,
                                                  int elem_bytes, const int *dims, int ndim,
                                                  int solvedim, char *out, size_t len) {
  if (kind == nullptr || (std::strcmp(kind, "solve") && std::strcmp(kind, "plan") &&
                          std::strcmp(kind, "refine")) ||
      (elem_bytes != 4 && elem_bytes != 8))
    return PENTAD_STATUS_INVALID_VALUE;
  penta::Shape sh;
  const char *why = "";
  pentadStatus_t st = penta::make_shape(dims, ndim, solvedim, sh, &why);
  if (st != PENTAD_STATUS_SUCCESS) return st;
  std::string gpu;
  if (gpu_name != nullptr) {
    gpu = gpu_name;
  } else {
    Context *ctx = penta::resolve(nullptr);
    if (!ctx->init()) return PENTAD_STATUS_NOT_INITIALIZED;
    gpu = ctx->gpu_name;
  }
  const int dir = std::strcmp(kind, "solve") ? (solvedim == 0 ? 0 : 1) : sh.dir;
  return penta::copy_out(penta::tune_key(gpu, kind, (size_t)elem_bytes, dir, sh.L.n, sh.L.n_sys),
                         out, len)
             ? PENTAD_STATUS_SUCCESS
             : PENTAD_STATUS_INVALID_VALUE;
}

extern "C" pentadStatus_t pentadsolver_autotune_solve(
    pentadsolver_handle_t h, int elem_bytes, const void *ds, const void *dl, const void *d,
    const void *du, const void *dw, void *x, void *x_save, const int *t_dims, int t_ndim,
    int t_solvedim, void *t_buffer, size_t t_buffer_bytes, int reps, void *stream,
    char *report, size_t report_len) {
  if ((elem_bytes != 4 && elem_bytes != 8) || !ds || !dl || !d || !du || !dw || !x)
    return PENTAD_STATUS_INVALID_VALUE;
  Context *ctx = penta::resolve(h);
  const char *why = "";
  std::string rep;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  pentadStatus_t st =
      elem_bytes == 8
          ? penta::autotune_solve<double>(
                *ctx, static_cast<const double *>(ds), static_cast<const double *>(dl),
                static_cast<const double *>(d), static_cast<const double *>(du),
                static_cast<const double *>(dw), static_cast<double *>(x),
                static_cast<double *>(x_save), t_dims, t_ndim, t_solvedim, t_buffer,
                t_buffer_bytes, reps, s, rep, &why)
          : penta::autotune_solve<float>(
                *ctx, static_cast<const float *>(ds), static_cast<const float *>(dl),
                static_cast<const float *>(d), static_cast<const float *>(du),
                static_cast<const float *>(dw), static_cast<float *>(x),
                static_cast<float *>(x_save), t_dims, t_ndim, t_solvedim, t_buffer,
                t_buffer_bytes, reps, s, rep, &why);
  if (st != PENTAD_STATUS_SUCCESS) {
    if (penta::env_flag("PENTA_DEBUG_LAUNCH")) std::fprintf(stderr, "[penta] autotune: %s\n", why);
    return st;
  }
  return penta::copy_out(rep, report, report_len) ? PENTAD_STATUS_SUCCESS
                                                  : PENTAD_STATUS_INVALID_VALUE;
}

extern "C" pentadStatus_t pentadsolver_autotune_plan(pentadsolver_plan_t plan, int reps,
                                                     void *stream, int *best_ctas) {
  if (plan == nullptr || plan->p == nullptr || reps < 1 || reps > 1000)
    return PENTAD_STATUS_INVALID_VALUE;
  penta::Plan &p = *plan->p;
  Context &ctx = *p.ctx;
  const char *why = "";
  if (!penta::on_own_device(ctx, &why)) return PENTAD_STATUS_INVALID_VALUE;
  penta::Plan &launching = p.fp32 ? *p.fp32 : p;  // whose ctas the launches use
  const int before = launching.ctas;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  static constexpr double kFractions[] = {1.0, 0.9, 0.75, 0.5};
  int best = before;
  float best_ms = -1.f;
  pentadStatus_t st = PENTAD_STATUS_SUCCESS;
  for (double f : kFractions) {
    launching.ctas = std::max(1, (int)(ctx.sm_count * f));
    if (p.fp32q) p.fp32q->ctas = launching.ctas;
    if ((st = pentadsolver_plan_execute(plan, stream)) != PENTAD_STATUS_SUCCESS) break;  // warm-up
    bool ok = cudaEventRecord(e0, static_cast<cudaStream_t>(stream)) == cudaSuccess;
    for (int r = 0; ok && r < reps; ++r) ok = pentadsolver_plan_execute(plan, stream) == PENTAD_STATUS_SUCCESS;
    float ms = 0.f;
    ok = ok && cudaEventRecord(e1, static_cast<cudaStream_t>(stream)) == cudaSuccess &&
         cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      st = PENTAD_STATUS_EXECUTION_FAILED;
      break;
    }
    ms /= reps;
    if (best_ms < 0.f || ms < best_ms) {
      best_ms = ms;
      best = launching.ctas;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  launching.ctas = st == PENTAD_STATUS_SUCCESS ? best : before;
  if (p.fp32q) p.fp32q->ctas = launching.ctas;
  if (st != PENTAD_STATUS_SUCCESS) return st;
  penta::TuneChoice c;
  c.ctas = best;
  c.ms = best_ms;
  penta::tune_store(p.tkey, c);
  if (best_ctas) *best_ctas = best;
  return PENTAD_STATUS_SUCCESS;
}
