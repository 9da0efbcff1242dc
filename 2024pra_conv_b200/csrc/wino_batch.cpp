// Batched persistent launch, schedule configurations and the autotuner.
//
// A batch holds the uneven 3x3 conv layers of a network (each with its own
// input, cached U, output and XB workspace).  Running it issues the input
// pre-pass of every layer that uses one and then ONE persistent fused-kernel
// launch whose CTAs walk the concatenated work blocks of all layers through
// a device-resident layer table; the whole sequence can be captured into a
// CUDA graph and replayed.  The reference has no counterpart: its harness
// runs one hard-wired shape per launch sequence (src/main.cpp:105-124,
// src/conv2d.cpp:458-494).
//
// The autotuner times every schedule configuration of every layer (CFG_*
// bits of wino_batch.h) with CUDA events, keeps the fastest per layer, then
// times whole-batch launches under three layer orders and keeps the fastest.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>
#include <cuda_runtime.h>

#include "winoconv.h"
#include "wino_param.h"
#include "wino_batch.h"


extern "C" {
int wino_fused_launch_variant(int variant, const wino::KernelParam* p, const wino::VariantArgs* va,
                              int cfg, unsigned grid, cudaStream_t stream);
int wino_fused_launch_batch(const void* table_dev, long long total_blocks, unsigned grid,
                            cudaStream_t stream);
int wino_launch_xb_layout(const wino::KernelParam* p, cudaStream_t stream);
int wino_fused_prepare_batch();
int wino_fused_prepare_variant(int variant);
size_t wino_xb_bytes(int n, int c, int h, int w);
long long wino_xb_items(int n, int c, int h, int w);
long long wino_fused_nblocks(int n, int h, int w, int k);
long long wino_fused_nblocks_cfg(int n, int c, int h, int w, int k, int cfg);
int wino_fused_cfg_splits(int c, int cfg);
int wino_launch_y32_to_f16(const float* y32, void* y, long long count, cudaStream_t stream);
int wino_launch_u_to_u2(const void* u, void* u2, int K, int C, cudaStream_t stream);
size_t wino_twostage_workspace_bytes(int n, int c, int h, int w, int k);
int wino_twostage_stage(int stage, const void* x, const void* ucache2, void* workspace, void* y, int n, int c,
                        int h, int w, int k, void* stream);
}

namespace {

using wino::BatchTable;
using wino::KernelParam;
using wino::LayerDesc;

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    return 148;
  return n;
}

KernelParam layer_param(const void* x, const void* ucache, void* xb, void* y, int n, int c, int h,
                        int w, int k) {
  KernelParam p;
  std::memset(&p, 0, sizeof(p));
  p.pin = const_cast<void*>(x);
  p.pout = y;
  p.transform_pin = xb;
  p.transform_filter = const_cast<void*>(ucache);
  p.n = (short)n; p.c = (short)c; p.h = (short)h; p.w = (short)w; p.k = (short)k;
  p.r = 3; p.s = 3; p.u = 1; p.v = 1; p.p = 1; p.q = 1;
  p.Oh = (short)h; p.Ow = (short)w;
  return p;
}

unsigned grid_for(long long blocks) {
  const long long sms = sm_count();
  return (unsigned)std::max<long long>(1, std::min(blocks, sms));
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace of a configuration: the XB records (unless direct), then the
// fp32 partial-sum output of split configurations.
size_t cfg_workspace_bytes(int n, int c, int h, int w, int k, int cfg) {
  size_t b = (cfg & wino::CFG_DIRECT) ? 0 : align256(wino_xb_bytes(n, c, h, w));
  if (wino_fused_cfg_splits(c, cfg) > 1) b += (size_t)n * k * h * w * sizeof(float);
  return b;
}

// One layer with a schedule configuration: zero the fp32 sums (split), the
// pre-pass (unless direct), the fused kernel, the fp16 rounding (split).
// `ws` holds cfg_workspace_bytes(..., cfg) bytes (may be null for a
// direct, unsplit configuration).
int run_layer_cfg(const KernelParam& p0, void* ws, int cfg, cudaStream_t s) {
  KernelParam p = p0;
  if (!ws) cfg = (cfg | wino::CFG_DIRECT) & ~(3 << wino::CFG_SPLIT_SHIFT);
  uint8_t* w8 = static_cast<uint8_t*>(ws);
  const bool split = wino_fused_cfg_splits(p.c, cfg) > 1;
  const long long ycount = (long long)p.n * p.k * p.h * p.w;
  p.transform_pin = (cfg & wino::CFG_DIRECT) ? nullptr : w8;
  p.mid_result = nullptr;
  if (split) {
    float* y32 = reinterpret_cast<float*>(
        w8 + ((cfg & wino::CFG_DIRECT) ? 0 : align256(wino_xb_bytes(p.n, p.c, p.h, p.w))));
    p.mid_result = y32;
    if (cudaMemsetAsync(y32, 0, (size_t)ycount * sizeof(float), s) != cudaSuccess) return WINO_ECUDA;
  }
  if (p.transform_pin && wino_launch_xb_layout(&p, s) != 0) return WINO_ECUDA;
  const long long nb = wino_fused_nblocks_cfg(p.n, p.c, p.h, p.w, p.k, cfg);
  if (wino_fused_launch_variant(WINO_VAR_F16, &p, nullptr, cfg, grid_for(nb), s) != 0) return WINO_ECUDA;
  if (split && wino_launch_y32_to_f16(static_cast<const float*>(p.mid_result), p.pout, ycount, s) != 0)
    return WINO_ECUDA;
  return WINO_OK;
}

// Mean microseconds of `fn` over `reps` launches after one warm-up, on `s`.
template <typename F>
int time_us(F&& fn, int reps, cudaStream_t s, float* us) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return WINO_ECUDA;
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return WINO_ECUDA;
  }
  int rc = fn();
  if (rc == WINO_OK) {
    cudaEventRecord(a, s);
    for (int i = 0; i < reps && rc == WINO_OK; ++i) rc = fn();
    cudaEventRecord(b, s);
    if (cudaEventSynchronize(b) != cudaSuccess) rc = WINO_ECUDA;
    float ms = 0.f;
    if (rc == WINO_OK && cudaEventElapsedTime(&ms, a, b) != cudaSuccess) rc = WINO_ECUDA;
    if (rc == WINO_OK) *us = ms * 1000.f / (float)std::max(reps, 1);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

// Route of a batch layer: inside the persistent fused launch (its tile
// blocks of 128 output channels x 32 tiles), or the two-stage path (tap GEMM
// units of 128 tiles x 256 output channels with full-width MMAs, M through
// a batch-owned workspace) launched before it.
constexpr int ROUTE_FUSED = 0, ROUTE_TWOSTAGE = 1;

struct Layer {
  KernelParam p;
  int cfg = 0;
  int route = ROUTE_FUSED;
  long long blocks = 0;
  float tuned_us = 0.f;     // fastest fused configuration alone
  float twostage_us = -1.f; // the two-stage route alone (-1: not timed or not applicable)
  void* u2 = nullptr;       // U in the two-stage GEMM's layout (batch-owned)
  void* ws2 = nullptr;      // two-stage workspace (batch-owned)
  // U2 and the workspace for the two-stage route, made on first use from the
  // layer's fused U cache (synchronous: not inside a stream capture)
  int ensure_twostage() {
    if (u2 && ws2) return WINO_OK;
    const size_t wsb = wino_twostage_workspace_bytes(p.n, p.c, p.h, p.w, p.k);
    if (wsb == 0) return WINO_EUNSUPPORTED;
    if (!u2 && cudaMalloc(&u2, (size_t)16 * p.k * p.c * 2) != cudaSuccess) return WINO_ECUDA;
    if (!ws2 && cudaMalloc(&ws2, wsb) != cudaSuccess) return WINO_ECUDA;
    if (wino_launch_u_to_u2(p.transform_filter, u2, p.k, p.c, nullptr) != 0) return WINO_ECUDA;
    return cudaDeviceSynchronize() == cudaSuccess ? WINO_OK : WINO_ECUDA;
  }
  int run_twostage(cudaStream_t s) const {
    for (int stage = 0; stage < 3; ++stage) {
      const int rc = wino_twostage_stage(stage, p.pin, u2, ws2, p.pout, p.n, p.c, p.h, p.w, p.k, s);
      if (rc != WINO_OK) return rc;
    }
    return WINO_OK;
  }
  void release() {
    if (u2) cudaFree(u2);
    if (ws2) cudaFree(ws2);
    u2 = ws2 = nullptr;
  }
};

struct Batch {
  std::vector<Layer> layers;
  std::vector<int> order;        // table order of the layers
  BatchTable* table_dev = nullptr;
  long long total = 0;
  bool dirty = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // Completion of the last run or graph launch, recorded on the caller's
  // stream.  commit() and destroy wait for it before they rewrite or free
  // the device table (or destroy the graph) that launch may still be reading:
  // a caller's non-blocking stream is not ordered against the synchronous
  // table copy on the legacy stream.
  cudaEvent_t done = nullptr;
  bool pending = false;

  int mark(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return WINO_ECUDA;
    if (cs != cudaStreamCaptureStatusNone) return WINO_OK;  // recorded by the replay's owner
    if (!done && cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess) return WINO_ECUDA;
    if (cudaEventRecord(done, s) != cudaSuccess) return WINO_ECUDA;
    pending = true;
    return WINO_OK;
  }

  int settle() {
    if (!pending) return WINO_OK;
    pending = false;
    return cudaEventSynchronize(done) == cudaSuccess ? WINO_OK : WINO_ECUDA;
  }

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }

  // Build the table in `order` and copy it to the device (synchronous: never
  // called inside a stream capture).
  int commit() {
    if (!dirty) return WINO_OK;
    if (!table_dev && cudaMalloc(&table_dev, sizeof(BatchTable)) != cudaSuccess) return WINO_ECUDA;
    BatchTable t;
    std::memset(&t, 0, sizeof(t));
    long long begin = 0;
    int nt = 0;
    for (size_t i = 0; i < order.size(); ++i) {
      const Layer& L = layers[order[i]];
      if (L.route != ROUTE_FUSED) continue;     // launched on its own before the table
      LayerDesc& d = t.layer[nt++];
      d.p = L.p;
      int cfg = L.cfg;
      if (!d.p.transform_pin) cfg |= wino::CFG_DIRECT;
      if (cfg & wino::CFG_DIRECT) d.p.transform_pin = nullptr;
      d.cfg = cfg;
      d.block_begin = begin;
      begin += L.blocks;
    }
    t.nlayers = nt;
    t.total = begin;
    total = begin;
    if (settle() != WINO_OK) return WINO_ECUDA;  // no launch still reads the old table
    if (cudaMemcpy(table_dev, &t, sizeof(t), cudaMemcpyHostToDevice) != cudaSuccess) return WINO_ECUDA;
    dirty = false;
    drop_graph();
    return WINO_OK;
  }

  int run(cudaStream_t s) {
    if (dirty) return WINO_EINVAL;  // commit first (outside any capture)
    for (int li : order) {
      const Layer& L = layers[li];
      if (L.route == ROUTE_TWOSTAGE) {
        const int rc = L.run_twostage(s);
        if (rc != WINO_OK) return rc;
        continue;
      }
      if (L.p.transform_pin && !(L.cfg & wino::CFG_DIRECT) && wino_launch_xb_layout(&L.p, s) != 0)
        return WINO_ECUDA;
    }
    if (total == 0) return WINO_OK;           // every layer on the two-stage route
    return wino_fused_launch_batch(table_dev, total, grid_for(total), s) == 0 ? WINO_OK : WINO_ECUDA;
  }
};

Batch* as_batch(void* h) { return static_cast<Batch*>(h); }

}  // namespace

extern "C" {

size_t wino_fused_cfg_workspace_bytes(int n, int c, int h, int w, int k, int cfg) {
  if (cfg < 0 || cfg >= wino::NCFG || wino_check_shape(n, c, h, w, k) != WINO_OK) return 0;
  return cfg_workspace_bytes(n, c, h, w, k, cfg);
}

// Bytes that serve every configuration (the tuner's workspace).
size_t wino_fused_tune_workspace_bytes(int n, int c, int h, int w, int k) {
  size_t m = 0;
  for (int cfg = 0; cfg < wino::NCFG; ++cfg)
    m = std::max(m, wino_fused_cfg_workspace_bytes(n, c, h, w, k, cfg));
  return m;
}

int wino_conv2d_fused_cfg(const void* x, const void* ucache, void* workspace, void* y, int n, int c,
                          int h, int w, int k, int cfg, void* stream) {
  if (!x || !ucache || !y) return WINO_EINVAL;
  if (cfg < 0 || cfg >= wino::NCFG) return WINO_EINVAL;
  if (workspace && (reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return WINO_EINVAL;
  const int st = wino_check_shape(n, c, h, w, k);
  if (st != WINO_OK) return st;
  if (!workspace && cfg_workspace_bytes(n, c, h, w, k, cfg) != 0) return WINO_EINVAL;
  if (!(cfg & wino::CFG_DIRECT) && wino_xb_items(n, c, h, w) >= (1LL << 31)) return WINO_EUNSUPPORTED;
  return run_layer_cfg(layer_param(x, ucache, nullptr, y, n, c, h, w, k), workspace, cfg,
                       (cudaStream_t)stream);
}

// The tuning space: with a workspace every configuration without
// CFG_DIRECT (direct reads never win when the pre-pass is available);
// without one, the direct unsplit configurations.
int wino_tune_layer(const void* x, const void* ucache, void* workspace, void* y, int n, int c, int h,
                    int w, int k, int reps, float* us_out, int* best_cfg, void* stream) {
  if (!x || !ucache || !y || !us_out || !best_cfg) return WINO_EINVAL;
  const int st = wino_check_shape(n, c, h, w, k);
  if (st != WINO_OK) return st;
  if (workspace && (reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return WINO_EINVAL;
  const KernelParam p = layer_param(x, ucache, nullptr, y, n, c, h, w, k);
  const cudaStream_t s = (cudaStream_t)stream;
  int best = -1;
  for (int cfg = 0; cfg < wino::NCFG; ++cfg) {
    us_out[cfg] = -1.f;
    if (workspace ? (cfg & wino::CFG_DIRECT) != 0
                  : (!(cfg & wino::CFG_DIRECT) || wino::cfg_split_level(cfg) != 0))
      continue;
    // a split level that gives the same splits as a lower one is skipped
    if (wino::cfg_split_level(cfg) > 0 &&
        wino_fused_cfg_splits(c, cfg) == wino_fused_cfg_splits(c, cfg - (1 << wino::CFG_SPLIT_SHIFT)))
      continue;
    float us = 0.f;
    const int rc = time_us([&] { return run_layer_cfg(p, workspace, cfg, s); }, reps, s, &us);
    if (rc != WINO_OK) return rc;
    us_out[cfg] = us;
    if (best < 0 || us < us_out[best]) best = cfg;
  }
  *best_cfg = best;
  return WINO_OK;
}

int wino_batch_create(void** out) {
  if (!out) return WINO_EINVAL;
  *out = new (std::nothrow) Batch();
  return *out ? WINO_OK : WINO_EINVAL;
}

int wino_batch_destroy(void* h) {
  Batch* b = as_batch(h);
  if (!b) return WINO_EINVAL;
  b->settle();
  b->drop_graph();
  for (Layer& L : b->layers) L.release();
  if (b->table_dev) cudaFree(b->table_dev);
  if (b->done) cudaEventDestroy(b->done);
  delete b;
  return WINO_OK;
}

int wino_batch_add_layer(void* h, const void* x, const void* ucache, void* xb_ws, void* y, int n,
                         int c, int hh, int w, int k) {
  Batch* b = as_batch(h);
  if (!b || !x || !ucache || !y) return WINO_EINVAL;
  if ((int)b->layers.size() >= wino::BATCH_MAX) return WINO_EUNSUPPORTED;
  const int st = wino_check_shape(n, c, hh, w, k);
  if (st != WINO_OK) return st;
  if (xb_ws && ((reinterpret_cast<uintptr_t>(xb_ws) & 15) != 0 || wino_xb_items(n, c, hh, w) >= (1LL << 31)))
    return WINO_EINVAL;
  Layer L;
  L.p = layer_param(x, ucache, xb_ws, y, n, c, hh, w, k);
  L.blocks = wino_fused_nblocks(n, hh, w, k);
  L.cfg = xb_ws ? 0 : wino::CFG_DIRECT;
  b->order.push_back((int)b->layers.size());
  b->layers.push_back(L);
  b->dirty = true;
  return WINO_OK;
}

int wino_batch_num_layers(void* h) {
  Batch* b = as_batch(h);
  return b ? (int)b->layers.size() : -1;
}

int wino_batch_set_config(void* h, int layer, int cfg) {
  Batch* b = as_batch(h);
  if (!b || layer < 0 || layer >= (int)b->layers.size() || cfg < 0 || cfg >= wino::NCFG ||
      wino::cfg_split_level(cfg) != 0)
    return WINO_EINVAL;
  b->layers[layer].cfg = cfg;
  b->dirty = true;
  return WINO_OK;
}

int wino_batch_get_config(void* h, int layer, int* cfg) {
  Batch* b = as_batch(h);
  if (!b || !cfg || layer < 0 || layer >= (int)b->layers.size()) return WINO_EINVAL;
  *cfg = b->layers[layer].cfg;
  return WINO_OK;
}

int wino_batch_set_route(void* h, int layer, int route) {
  Batch* b = as_batch(h);
  if (!b || layer < 0 || layer >= (int)b->layers.size() || (route != ROUTE_FUSED && route != ROUTE_TWOSTAGE))
    return WINO_EINVAL;
  Layer& L = b->layers[layer];
  if (route == ROUTE_TWOSTAGE) {
    if (b->settle() != WINO_OK) return WINO_ECUDA;
    const int rc = L.ensure_twostage();
    if (rc != WINO_OK) return rc;
  }
  L.route = route;
  b->dirty = true;
  return WINO_OK;
}

int wino_batch_get_route(void* h, int layer, int* route, float* fused_us, float* twostage_us) {
  Batch* b = as_batch(h);
  if (!b || !route || layer < 0 || layer >= (int)b->layers.size()) return WINO_EINVAL;
  const Layer& L = b->layers[layer];
  *route = L.route;
  if (fused_us) *fused_us = L.tuned_us;
  if (twostage_us) *twostage_us = L.twostage_us;
  return WINO_OK;
}

int wino_batch_set_order(void* h, const int* order, int n) {
  Batch* b = as_batch(h);
  if (!b || !order || n != (int)b->layers.size()) return WINO_EINVAL;
  std::vector<int> o(order, order + n), sorted(o);
  std::sort(sorted.begin(), sorted.end());
  for (int i = 0; i < n; ++i)
    if (sorted[i] != i) return WINO_EINVAL;  // must be a permutation
  b->order = o;
  b->dirty = true;
  return WINO_OK;
}

int wino_batch_get_order(void* h, int* order, int n) {
  Batch* b = as_batch(h);
  if (!b || !order || n != (int)b->layers.size()) return WINO_EINVAL;
  std::copy(b->order.begin(), b->order.end(), order);
  return WINO_OK;
}

int wino_batch_commit(void* h) {
  Batch* b = as_batch(h);
  return b ? b->commit() : WINO_EINVAL;
}

int wino_batch_run(void* h, void* stream) {
  Batch* b = as_batch(h);
  if (!b || b->layers.empty()) return WINO_EINVAL;
  int rc = b->commit();
  if (rc != WINO_OK) return rc;
  rc = b->run((cudaStream_t)stream);
  return rc != WINO_OK ? rc : b->mark((cudaStream_t)stream);
}

// Autotune: per-layer configurations (exhaustive over CFG_*) and routes
// (the fused launch's 128 x 32 tile blocks or the two-stage path's 128 x 256
// tap-GEMM units, the faster alone), then the layer order of the table among
// {as added, longest first, longest/shortest interleaved}; the routes picked
// stay only if the whole batch beats the all-fused batch in the best order.
// layer_us: nlayers x NCFG timings (-1 = not applicable); order_us: the
// three whole-batch timings with the picked routes.  Leaves the best choice
// set; wino_batch_get_route reports each layer's route and both timings.
int wino_batch_tune(void* h, int reps, float* layer_us, float* order_us, void* stream) {
  Batch* b = as_batch(h);
  if (!b || b->layers.empty()) return WINO_EINVAL;
  const cudaStream_t s = (cudaStream_t)stream;
  const int nl = (int)b->layers.size();
  for (int i = 0; i < nl; ++i) {
    Layer& L = b->layers[i];
    float us[wino::NCFG];
    int best = 0;
    // batch layers run unsplit: time the configurations without splits
    best = -1;
    for (int cfg = 0; cfg < wino::NCFG; ++cfg) {
      us[cfg] = -1.f;
      if (wino::cfg_split_level(cfg) != 0) continue;
      if (!L.p.transform_pin && !(cfg & wino::CFG_DIRECT)) continue;
      float t = 0.f;
      const int rc = time_us([&] { return run_layer_cfg(L.p, L.p.transform_pin, cfg, s); }, reps, s, &t);
      if (rc != WINO_OK) return rc;
      us[cfg] = t;
      if (best < 0 || t < us[best]) best = cfg;
    }
    L.cfg = best;
    L.tuned_us = us[best];
    if (layer_us)
      for (int c = 0; c < wino::NCFG; ++c) layer_us[i * wino::NCFG + c] = us[c];
    // the two-stage route's tile shape (128 tiles x 256 output channels per
    // tap-GEMM unit), where the shape has one
    L.twostage_us = -1.f;
    if (wino_twostage_workspace_bytes(L.p.n, L.p.c, L.p.h, L.p.w, L.p.k) > 0) {
      const int rc = L.ensure_twostage();
      if (rc == WINO_OK) {
        float t = 0.f;
        const int rt = time_us([&] { return L.run_twostage(s); }, reps, s, &t);
        if (rt != WINO_OK) return rt;
        L.twostage_us = t;
      } else if (rc != WINO_EUNSUPPORTED) {
        return rc;
      }
    }
  }
  // routes: each layer the faster of its best fused configuration and the
  // two-stage route, measured alone
  std::vector<int> picked(nl, ROUTE_FUSED);
  for (int i = 0; i < nl; ++i) {
    const Layer& L = b->layers[i];
    if (L.twostage_us >= 0.f && L.twostage_us < L.tuned_us) picked[i] = ROUTE_TWOSTAGE;
    b->layers[i].route = picked[i];
  }
  std::vector<int> natural(nl), longest(nl), inter;
  std::iota(natural.begin(), natural.end(), 0);
  longest = natural;
  std::stable_sort(longest.begin(), longest.end(),
                   [&](int a, int c) { return b->layers[a].tuned_us > b->layers[c].tuned_us; });
  for (int lo = 0, hi = nl - 1; lo <= hi;) {
    inter.push_back(longest[lo++]);
    if (lo <= hi) inter.push_back(longest[hi--]);
  }
  const std::vector<int>* orders[3] = {&natural, &longest, &inter};
  int best_o = 0;
  float best_us = 0.f;
  for (int o = 0; o < 3; ++o) {
    b->order = *orders[o];
    b->dirty = true;
    int rc = b->commit();
    if (rc != WINO_OK) return rc;
    float us = 0.f;
    rc = time_us([&] { return b->run(s); }, reps, s, &us);
    if (rc != WINO_OK) return rc;
    if (order_us) order_us[o] = us;
    if (o == 0 || us < best_us) {
      best_us = us;
      best_o = o;
    }
  }
  b->order = *orders[best_o];
  // the fused launch overlaps its layers, so the picked routes are kept only
  // if the whole batch is faster with them than with every layer fused
  if (std::count(picked.begin(), picked.end(), ROUTE_TWOSTAGE) > 0) {
    for (Layer& L : b->layers) L.route = ROUTE_FUSED;
    b->dirty = true;
    int rc = b->commit();
    if (rc != WINO_OK) return rc;
    float all_fused = 0.f;
    rc = time_us([&] { return b->run(s); }, reps, s, &all_fused);
    if (rc != WINO_OK) return rc;
    if (best_us < all_fused)
      for (int i = 0; i < nl; ++i) b->layers[i].route = picked[i];
  }
  b->dirty = true;
  return b->commit();
}

// Capture one run (pre-passes + the persistent launch) into a CUDA graph.
// The capture uses a stream of its own (the legacy default stream cannot be
// captured); the graph may then be launched on any stream.  `stream` is
// accepted for symmetry and unused.
int wino_batch_graph_capture(void* h, void* stream) {
  (void)stream;
  Batch* b = as_batch(h);
  if (!b || b->layers.empty()) return WINO_EINVAL;
  int rc = b->commit();
  if (rc != WINO_OK) return rc;
  if (wino_fused_prepare_batch() != 0) return WINO_ECUDA;
  if (b->settle() != WINO_OK) return WINO_ECUDA;  // the old graph may still be running
  b->drop_graph();
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return WINO_ECUDA;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaStreamDestroy(s);
    return WINO_ECUDA;
  }
  rc = b->run(s);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  cudaStreamDestroy(s);
  if (rc != WINO_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc != WINO_OK ? rc : WINO_ECUDA;
  }
  if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    return WINO_ECUDA;
  }
  b->graph = g;
  return WINO_OK;
}

int wino_batch_graph_launch(void* h, void* stream) {
  Batch* b = as_batch(h);
  if (!b || !b->exec || b->dirty) return WINO_EINVAL;
  if (cudaGraphLaunch(b->exec, (cudaStream_t)stream) != cudaSuccess) return WINO_ECUDA;
  return b->mark((cudaStream_t)stream);
}

}  // extern "C"
