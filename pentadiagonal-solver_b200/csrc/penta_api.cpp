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
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>

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

// ---------------------------------------------------------------------------
// Contexts
// ---------------------------------------------------------------------------
struct Context {
  int device = -1;
  int sm_count = 0;
  int smem_optin = 0;  // max dynamic shared memory per block (bytes)
  std::mutex mu;
  Algo forced[3] = {Algo::Auto, Algo::Auto, Algo::Auto};
  int forced_lanes[3] = {0, 0, 0};
  std::atomic<const char *> ran[3] = {{kNone}, {kNone}, {kNone}};
  std::string variant[3];
  std::unordered_map<long long, int> occ_cache;  // (variant, n) -> CTAs/SM

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
    sm_count = sms;
    smem_optin = optin;
    device = dev;
    return true;
  }
};

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
  long long inner = 1, outer = 1;
  for (int k = 0; k < ndim; ++k) {
    if (dims[k] < 1) { *why = "a dimension is < 1"; return PENTAD_STATUS_INVALID_VALUE; }
    if (k < solvedim) inner *= dims[k];
    if (k > solvedim) outer *= dims[k];
  }
  const long long n = dims[solvedim];
  if (n <= 4) {
    // The reference asserts sys_size > 4 on every path (pentad_cuda.cu:1203).
    *why = "the solve dimension must be longer than 4";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  if (n > (1LL << 24) || inner * outer > (1LL << 40)) {
    *why = "grid too large";
    return PENTAD_STATUS_INVALID_VALUE;
  }
  sh.L.n = n;
  sh.L.inner = inner;
  sh.L.n_sys = inner * outer;
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
              int &occ_out) {
  if (!tma_supported<F>(a)) return false;
  // the scratch variants keep (dw2, x2) in the caller's buffer
  // (128-byte aligned: they drop whole 128-byte lines of it from L2)
  const bool scr_ok = a.scratch != nullptr &&
                      reinterpret_cast<uintptr_t>(a.scratch) % 128 == 0 &&
                      tma_scratch_bytes<F>(a.L) <= usable_buf;
  const std::vector<TmaConfig> &all = tma_configs<F>();
  // PENTA_TMA_VARIANT="R,stages,xstages,scratch" restricts the choice (tuning)
  int want[4] = {-1, -1, -1, -1};
  if (const char *e = std::getenv("PENTA_TMA_VARIANT"))
    std::sscanf(e, "%d,%d,%d,%d", &want[0], &want[1], &want[2], &want[3]);
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
// PENTA_TMEM_VARIANT="stages,xstages" restricts the choice (tuning).
template <typename F>
bool pick_tmem(Context &ctx, const SolveArgs<F> &a, bool contig, size_t usable_buf,
               TmemConfig &out) {
  bool w2s = false;
  if (!tmem_supported<F>(a, contig, usable_buf, w2s)) return false;
  int want[2] = {-1, -1};
  if (const char *e = std::getenv("PENTA_TMEM_VARIANT"))
    std::sscanf(e, "%d,%d", &want[0], &want[1]);
  const std::vector<TmemConfig> &all = tmem_configs<F>();
  for (size_t i = 0; i < all.size(); ++i) {
    const TmemConfig &c = all[i];
    if (c.contig != contig || c.w2s != w2s) continue;
    if ((want[0] >= 0 && c.stages != want[0]) || (want[1] >= 0 && c.xstages != want[1]))
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
template <typename F>
pentadStatus_t solve(Context &ctx, const F *ds, const F *dl, const F *d,
                     const F *du, const F *dw, F *x, const int *dims,
                     int ndim, int solvedim, void *buf, size_t buf_bytes,
                     cudaStream_t stream, const char **why) {
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
  int *status_word = device_status_word(ctx.device);
  if (status_word == nullptr) {
    *why = "cannot address the device status word";
    return PENTAD_STATUS_INTERNAL_ERROR;
  }
  SolveArgs<F> a{ds, dl, d, du, dw, x, sh.L, buf, buf_bytes, status_word};
  const int dir = sh.dir;
  const bool contig = (dir == 0);
  const Algo want = selected_algo(ctx, dir);
  const int lanes = selected_lanes(ctx, dir);
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
      if (!env_flag("PENTA_NO_TMA") && sf_tmem_supported<F>(a, contig, ctx.smem_optin)) {
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
      if (P == 2 && !env_flag("PENTA_NO_TMA") && !env_flag("PENTA_NO_TMEM")) {
        TmemConfig mc{};
        const size_t usable = std::min(buf_bytes, buffer_bytes(sh, sizeof(F)));
        if (pick_tmem<F>(ctx, a, contig, usable, mc)) {
          err = launch_tmem<F>(a, mc, ctx.sm_count, stream);
          if (err == cudaSuccess) {
            char vb[96];
            std::snprintf(vb, sizeof vb, "thomas-pcr:tmem P2 S16 R%d x%d/%d%s%s", mc.R,
                          mc.stages, mc.xstages, mc.w2s ? " w2s" : "",
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
      if (contig && P == 2 && !env_flag("PENTA_NO_TMA")) {
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
      if (!contig && P == 2 && !env_flag("PENTA_NO_TMA")) {
        TmaConfig tc{};
        int occ = 0;
        const size_t usable = std::min(buf_bytes, buffer_bytes(sh, sizeof(F)));
        if (pick_tma<F>(ctx, a, usable, tc, occ)) {
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

size_t size_query(const int *dims, int ndim, int solvedim, size_t elem) {
  Shape sh;
  const char *why = "";
  if (make_shape(dims, ndim, solvedim, sh, &why) != PENTAD_STATUS_SUCCESS)
    return 0;
  return buffer_bytes(sh, elem);
}

}  // namespace
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
  if (owned) delete c;
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
  int *word = penta::device_status_word(ctx->device);
  if (word == nullptr) return PENTAD_STATUS_INTERNAL_ERROR;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int host = 0;
  const int zero = 0;
  if (cudaMemcpyAsync(&host, word, sizeof(int), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(word, &zero, sizeof(int), cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  if (bits) *bits = host;
  return (host & penta::STATUS_ZERO_PIVOT_BIT) ? PENTAD_STATUS_ZERO_PIVOT
                                               : PENTAD_STATUS_SUCCESS;
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
