/*
 * Extension C-ABI of the B200 Winograd F(2x2,3x3) conv2d library
 * (libwinoconv.so).  Plain C types only; every pointer is device memory unless
 * stated otherwise; `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * The reference has no counterpart for these entry points beyond the plugin
 * ABI in conv2d.h (reference include/conv2d.h:69-70): they expose the pieces
 * that ABI hides (a one-shot filter transform whose result is reused across
 * calls, the fused conv on a cached U, the unfused comparator path) so that a
 * caller can keep U resident and so that tests and benchmarks can reach each
 * stage.  Each function cites the reference stage it implements.
 *
 * Shape contract (all Winograd entry points): 3x3 filter, stride 1, pad 1,
 * c % 16 == 0, k % 16 == 0, n, c, h, w, k in [1, 32767].  Other shapes:
 * wino_conv2d_direct, and getkernelInfo dispatches them there itself.
 * Return: 0 on success or one of the WINO_E* codes below.
 */
#ifndef WINO_WINOCONV_H
#define WINO_WINOCONV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WINO_OK = 0,
  WINO_EINVAL = 1,        /* null pointer or invalid argument            */
  WINO_EUNSUPPORTED = 2,  /* shape outside the contract above            */
  WINO_ECUDA = 3,         /* a CUDA runtime call failed                  */
  WINO_EDEVICE = 4,       /* a kernel reported an error (see error word) */
  WINO_ESCRATCH = 5,      /* scratch or caller workspace too small for the shape */
  WINO_ESTALE = 6,        /* persisted U cache is for other weights, shape or layout */
  WINO_EIO = 7            /* file could not be read or written */
};

/* Precision variants of the GEMM stage. */
enum {
  WINO_VAR_F16 = 0,       /* fp16 operands, fp32 accumulate              */
  WINO_VAR_BF16 = 1,      /* bf16 operands, fp32 accumulate              */
  WINO_VAR_F8 = 2,        /* fp8 e4m3 operands with per-channel scales   */
  WINO_VAR_F16_HILO = 3   /* fp16 with the U residual as a second GEMM   */
};

/* Validate a problem against the shape contract (no CUDA calls). */
int wino_check_shape(int n, int c, int h, int w, int k);

/* The route getkernelInfo takes for a problem_t (conv2d.h), without CUDA
 * calls: the direct kernel (no transform_filter, or a shape outside the
 * Winograd contract whose re-laid-out weights do not fit it), the fused
 * kernel reading the NCHW input (no usable transform_pin), the fused kernel
 * after the input pre-pass, the two-stage route (pre-pass, input-fused tap
 * GEMM with M in mid_result, output transform: needs mid_result of
 * 4*k*h*w*n fp16 to hold 16*k*tiles, i.e. even h and w), or the tensor-core
 * implicit GEMM for shapes outside the Winograd contract (weights re-laid
 * out into transform_filter, which must hold wino_igemm_weight_bytes).
 * Returns a WINO_ROUTE_* value, or minus a WINO_E* code for an invalid
 * problem. */
enum {
  WINO_ROUTE_DIRECT = 0,
  WINO_ROUTE_FUSED = 1,
  WINO_ROUTE_FUSED_XB = 2,
  WINO_ROUTE_TWOSTAGE = 3,
  WINO_ROUTE_IGEMM = 4
};
int wino_dropin_route(const void* problem);

/* Bytes of the U cache for a variant (fp16: 16*k*c*2). */
size_t wino_ucache_bytes(int k, int c, int variant);

/* Filter transform U = G g G^T of fp16 KCRS weights into the tile-major
 * fp16 U cache (reference src/preprocessing.cuh:75-270, GgGT*).  One-shot:
 * the result stays valid for as long as the weights do. */
int wino_filter_transform(const void* weight, void* ucache, int k, int c, void* stream);

/* Persistence of the fp16 U cache across calls and processes (the reference
 * re-runs its filter transform on every iteration, src/main.cpp:121):
 * wino_weight_tag computes a 64-bit content tag of fp16 KCRS weights on the
 * GPU (synchronises `stream`); wino_ucache_save writes a U cache with its
 * shape, layout version and that tag; wino_ucache_load fills a caller's U
 * buffer from such a file and returns WINO_ESTALE -- leaving the buffer
 * untouched -- when the file belongs to other weights (tag), another shape or
 * another layout version, so a caller re-runs wino_filter_transform then.
 * wino_ucache_save copies U with a synchronous copy on the legacy default
 * stream: the stream that wrote U must be synchronised first when it is a
 * non-blocking stream.  wino_ucache_load returns once the U buffer is
 * complete on the device. */
int wino_weight_tag(const void* weight, int k, int c, unsigned long long* tag, void* stream);
int wino_ucache_save(const char* path, const void* ucache, int k, int c, unsigned long long tag);
int wino_ucache_load(const char* path, void* ucache, int k, int c, unsigned long long tag);

/* Fused conv on a prepared fp16 U cache: input transform, tensor-core tap
 * GEMMs and output transform in one persistent kernel (reference
 * src/preprocessing.cuh:273-424, src/matrixmul.cuh:139-556,
 * src/conv2d.cpp:17-250).  x: NCHW fp16, y: N K H W fp16. */
int wino_conv2d_fused(const void* x, const void* ucache, void* y, int n, int c, int h, int w,
                      int k, void* stream);

/* The same with a caller workspace of wino_fused_workspace_bytes() bytes
 * (16-byte aligned): a pre-pass writes the input there once in a
 * channel-blocked layout, which the fused kernel stages into shared memory
 * with bulk copies -- the fast path.  (The reference likewise hands its
 * input-transform kernel the caller's transform_pin workspace,
 * src/main.cpp:36-38, src/preprocessing.cuh:273-424.) */
size_t wino_fused_workspace_bytes(int n, int c, int h, int w);
/* The pre-pass alone (input -> workspace), e.g. to time it apart. */
int wino_input_layout(const void* x, void* workspace, int n, int c, int h, int w, void* stream);
int wino_conv2d_fused_ws(const void* x, const void* ucache, void* workspace, void* y, int n, int c,
                         int h, int w, int k, void* stream);

/* The fast path with the step that follows a conv in a ResNet block folded
 * into its output transform (the reference stops at the conv, writing M and
 * transforming it in a separate kernel, src/conv2d.cpp:17-250):
 *   y = relu ? max(conv(x) + bias[k] + residual, 0) : conv(x) + bias[k] + residual
 * bias: fp32 per output channel, or NULL; residual: fp16 in y's N K H W
 * layout (4-byte aligned, may be y itself), or NULL.  conv + bias is
 * rounded to fp16 before the residual is added (in fp32) and the result
 * rounded again.  workspace as for wino_conv2d_fused_ws. */
int wino_conv2d_fused_epilogue(const void* x, const void* ucache, void* workspace, void* y,
                               const float* bias, const void* residual, int relu, int n, int c, int h,
                               int w, int k, void* stream);

/* Direct convolution for any filter size r x s, stride (u, v) and padding
 * (p, q) and any channel counts (implicit GEMM on CUDA cores, fp32
 * accumulation); y: N K OH OW with OH = (h - r + 2p)/u + 1, OW likewise.
 * getkernelInfo dispatches every shape outside the Winograd contract here
 * (the reference ignores r, s, u, v, p, q, src/conv2d.cpp:254-271). */
int wino_conv2d_direct(const void* x, const void* weight, void* y, int n, int c, int h, int w, int k,
                       int r, int s, int u, int v, int p, int q, void* stream);

/* Implicit-GEMM convolution on the tcgen05 tensor cores for the same general
 * shapes (any r x s, stride, padding; channel counts padded to 16 with
 * zeros): D[pixel][k] over K-steps of (tap, 16 channels), fp16 operands,
 * fp32 accumulation, one fp16 rounding of y.  wino_igemm_weight_transform
 * re-lays the KCRS weights into wprep (wino_igemm_weight_bytes bytes,
 * 16-byte aligned: the operand, then a 128-byte slot for the input's TMA
 * tensor map, used when wprep is 64-byte aligned), whose operand stays
 * valid for as long as the weights do;
 * wino_conv2d_igemm reads the pixel operand straight from the NCHW input
 * (1x1 / stride 1 / pad 0 layers with h*w % 64 == 0 and k > 128 through a
 * tensor map it writes to wprep's slot in stream order, so one wprep serves
 * one stream at a time).  getkernelInfo takes this route for shapes outside
 * the Winograd contract when the operand fits the caller's transform_filter
 * (16*k*c fp16, reference src/main.cpp:38), i.e. r*s*ceil(c/16)*round16(k)
 * <= k*c. */
size_t wino_igemm_weight_bytes(int c, int k, int r, int s);
int wino_igemm_weight_transform(const void* weight, void* wprep, int k, int c, int r, int s,
                                void* stream);
int wino_conv2d_igemm(const void* x, const void* wprep, void* y, int n, int c, int h, int w, int k,
                      int r, int s, int u, int v, int p, int q, void* stream);

/* The plain unfused path, the comparator of the fused kernel: input
 * transform to V in global memory, the 16 tap GEMMs as one batched tcgen05
 * GEMM writing M (fp16) to global memory, output transform -- the stage
 * structure of the reference pipeline (src/preprocessing.cuh:273-424,
 * src/matrixmul.cuh:139-556, src/conv2d.cpp:17-250).  It reads U in its own
 * layout, made by wino_filter_transform_unfused; v_ws and m_ws are caller
 * workspaces of the sizes wino_unfused_workspace_bytes reports. */
int wino_filter_transform_unfused(const void* weight, void* ucache2, int k, int c, void* stream);
int wino_unfused_workspace_bytes(int n, int c, int h, int w, int k, size_t* v_bytes,
                                 size_t* m_bytes);
int wino_conv2d_unfused(const void* x, const void* ucache2, void* y, void* v_ws, void* m_ws, int n,
                        int c, int h, int w, int k, void* stream);

/* Conv with a precision variant of the GEMM stage (WINO_VAR_*), everything
 * per call: the variant's filter transform (bf16 U; U_hi + U_lo; or fp8 U
 * with the input's per-channel scales folded in and per-(tap, k) scales),
 * the input pre-pass (for fp8 also the per-channel max |x|), then the fused
 * kernel of the variant.  workspace: wino_variant_workspace_bytes() bytes,
 * 256-byte aligned.  fp8 needs c % 32 == 0.  x: NCHW fp16, weight: KCRS
 * fp16, y: N K H W fp16.  (The reference computes in fp16 only,
 * src/matrixmul.cuh:28-35; these variants have no counterpart there.) */
size_t wino_variant_workspace_bytes(int variant, int n, int c, int h, int w, int k);
int wino_conv2d_variant(int variant, const void* x, const void* weight, void* y, void* workspace,
                        int n, int c, int h, int w, int k, void* stream);

/* Two-stage F(2x2,3x3): an input pre-pass, full-width tcgen05 tap GEMMs
 * (one tap x 128 tiles x 256 output channels per work unit), M is
 * written as fp16 (16 * k * tiles elements, tiles = n * ceil(h/2) *
 * ceil(w/2)) and a third kernel applies the output transform.  For c <= 256
 * the pre-pass writes the transformed tiles V (16 * tiles8 * c fp16, tiles8
 * = tiles rounded up to 8) and the GEMM keeps each CTA's U resident and reads
 * V by bulk copy; for c > 256 the pre-pass writes the channel-blocked input
 * and the GEMM forms V in shared memory and streams U.  ucache2: U in the
 * unfused GEMM layout (wino_filter_transform_unfused).  workspace: 256-byte
 * aligned, wino_twostage_workspace_bytes() bytes (pre-pass output, then M).
 * The output equals the unfused comparator's (same operands and rounding
 * points); the reference's pipeline writes V and M to its workspaces the same
 * way (src/preprocessing.cuh:273-424, src/matrixmul.cuh:139-556).
 * getkernelInfo takes this route when M fits the caller's mid_result
 * (4*k*h*w*n fp16: even h and w) and the pre-pass output fits transform_pin.
 * Shapes whose blocked-input record block (one image, 16 channels) reaches
 * 2^31 bytes return WINO_EUNSUPPORTED (workspace size 0). */
size_t wino_twostage_workspace_bytes(int n, int c, int h, int w, int k);
int wino_conv2d_twostage(const void* x, const void* ucache2, void* workspace, void* y, int n, int c,
                         int h, int w, int k, void* stream);
/* One stage of it: 0 input pre-pass, 1 tap GEMM, 2 output transform. */
int wino_twostage_stage(int stage, const void* x, const void* ucache2, void* workspace, void* y,
                        int n, int c, int h, int w, int k, void* stream);

/* The same two-stage F(2x2,3x3) with an fp8 e4m3 tensor-core GEMM.  hilo
 * 1: U and V are each split into e4m3 hi + lo terms (hi = e4m3(v), lo =
 * e4m3(v - hi)) and the GEMM accumulates hi.hi + lo.hi + hi.lo with
 * kind::f8f6f4 MMAs, 32 channels per step -- fp16-level accuracy; hilo 0:
 * single e4m3 terms, one MMA per step and half the transformed-tile bytes
 * -- faster, at single-term fp8 accuracy.  Scales: per input
 * channel from its max |x| (|V| <= 4 max|x_c|, folded into U) and per (tap,
 * output channel) on U, applied before M is rounded to fp16.  Launches a
 * channel-max pass, the U split, the V split (transformed tiles), the GEMM
 * and the output transform.  ucache2: the fp16 U in the unfused layout
 * (wino_filter_transform_unfused).  c a multiple of 32, at most 256;
 * workspace 256-byte aligned, wino_twostage_f8_workspace_bytes() bytes (0:
 * shape not supported).  The reference computes in fp16 only
 * (src/matrixmul.cuh:28-35); this variant has no counterpart there. */
size_t wino_twostage_f8_workspace_bytes(int n, int c, int h, int w, int k, int hilo);
int wino_conv2d_twostage_f8(const void* x, const void* ucache2, void* workspace, void* y, int n, int c,
                            int h, int w, int k, int hilo, void* stream);

/* Winograd F(4x4,3x3) (36 taps, 4x4 output tiles; no counterpart in the
 * reference, which has F(2x2,3x3) only: src/preprocessing.cuh:75-424,
 * src/matrixmul.cuh:139-556, src/conv2d.cpp:17-250).  U and V are formed in
 * fp32 and stored as fp16: one piece (hilo = 0) or a hi + lo pair (hilo = 1,
 * products hi*hi + lo*hi + hi*lo accumulated in fp32); M stays fp32 and the
 * output transform is fp32.  Same shape contract as the fused path (3x3,
 * stride 1, pad 1, c and k multiples of 16).  workspace: 256-byte aligned,
 * wino_f4_workspace_bytes() bytes; its first wino_f4_filter_bytes() bytes
 * hold the transformed filter, written by wino_f4_filter_transform() once
 * per weight tensor and read by every wino_conv2d_f4() after it (the rest
 * holds V and M).  Too small a workspace returns WINO_ESCRATCH. */
size_t wino_f4_filter_bytes(int k, int c, int hilo);
size_t wino_f4_workspace_bytes(int n, int c, int h, int w, int k, int hilo);
int wino_f4_filter_transform(const void* weight, int k, int c, int hilo, void* workspace,
                             size_t workspace_bytes, void* stream);
int wino_conv2d_f4(const void* x, void* y, int n, int c, int h, int w, int k, int hilo,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Schedule configurations of the fused kernel (bits): WINO_CFG_KMAJOR orders
 * the work blocks k-block-major (consecutive blocks share U) instead of
 * tile-major (they share input tiles); WINO_CFG_DIRECT makes the producers
 * read the NCHW input directly instead of the pre-pass workspace; bits 2-3
 * (WINO_CFG_SPLIT(L)) split each block's 16-channel steps over up to 4^L CTAs
 * that add fp32 partial outputs, rounded to fp16 by a second pass -- for
 * layers with too few blocks to fill the GPU.  Unsplit configurations
 * compute bit-identical results; split ones differ only in the fp32
 * summation order. */
enum { WINO_CFG_KMAJOR = 1, WINO_CFG_DIRECT = 2, WINO_CFG_SPLIT_SHIFT = 2, WINO_NCFG = 16 };
#define WINO_CFG_SPLIT(level) ((level) << WINO_CFG_SPLIT_SHIFT)

/* Workspace of one configuration (pre-pass records unless direct, then the
 * fp32 sums of split configurations; 0 = none needed) and the size that
 * serves every configuration (for wino_tune_layer). */
size_t wino_fused_cfg_workspace_bytes(int n, int c, int h, int w, int k, int cfg);
size_t wino_fused_tune_workspace_bytes(int n, int c, int h, int w, int k);

/* One fp16 conv on a cached U with a schedule configuration; workspace:
 * wino_fused_cfg_workspace_bytes() bytes, 256-byte aligned (NULL allowed
 * when that is 0). */
int wino_conv2d_fused_cfg(const void* x, const void* ucache, void* workspace, void* y, int n, int c,
                          int h, int w, int k, int cfg, void* stream);

/* Exhaustive tuning of one layer: mean microseconds of every configuration
 * of the tuning space (us_out[WINO_NCFG], -1 for configurations outside it)
 * over `reps` runs after one warm-up, and the fastest in *best_cfg.  With a
 * workspace (wino_fused_tune_workspace_bytes) the space is every
 * configuration without WINO_CFG_DIRECT, split levels that give the same
 * number of splits as a lower one left out; without one, the two direct
 * unsplit configurations.  Synchronises `stream`; not inside a capture. */
int wino_tune_layer(const void* x, const void* ucache, void* workspace, void* y, int n, int c, int h,
                    int w, int k, int reps, float* us_out, int* best_cfg, void* stream);

/* Batched persistent launch (no counterpart in the reference, whose harness
 * runs one hard-wired shape per launch sequence, src/main.cpp:105-124).  A
 * batch holds up to 32 fp16 layers, each with its input, cached U, output
 * and (optional) pre-pass workspace; wino_batch_run issues the pre-passes and
 * ONE persistent fused-kernel launch over all layers' work blocks (a device
 * layer table); wino_batch_graph_capture records that sequence in a CUDA
 * graph, wino_batch_graph_launch replays it.  Batch layers run unsplit.
 * wino_batch_tune runs the autotuner: per layer the route (fused or
 * two-stage, kept only if the whole batch is faster with the picks than
 * all-fused) and the fastest unsplit
 * configuration (exhaustive), then the
 * fastest table order among {as added, longest first, longest/shortest
 * interleaved}; layer_us receives nlayers x WINO_NCFG timings, order_us the
 * three whole-batch timings (either may be NULL).  Configuration and order
 * changes invalidate a captured graph.  wino_batch_run and
 * wino_batch_graph_launch record their completion on the caller's stream;
 * the next commit (explicit, or the one a run or capture after a change
 * makes) waits for it on the host before it rewrites the device layer table,
 * so an earlier launch on any stream never reads a half-rewritten table.  Each layer needs its own workspace
 * (wino_fused_workspace_bytes of its shape, or NULL for direct reads): the
 * pre-passes of a run write all workspaces before the one launch reads
 * them, so layers sharing one would overwrite each other. */
int wino_batch_create(void** batch);
int wino_batch_destroy(void* batch);
int wino_batch_add_layer(void* batch, const void* x, const void* ucache, void* workspace, void* y,
                         int n, int c, int h, int w, int k);
int wino_batch_num_layers(void* batch);
int wino_batch_set_config(void* batch, int layer, int cfg);
int wino_batch_get_config(void* batch, int layer, int* cfg);
/* Route of a batch layer (a tile-shape choice): 0 inside the persistent
 * fused launch (128 output channels x 32 tiles per block), 1 the two-stage
 * path (tap-GEMM units of 128 tiles x 256 output channels, M in a
 * batch-owned workspace, U relaid from the layer's fused U cache) launched
 * before it.  Setting route 1 allocates those buffers (outside any stream
 * capture).  get_route also reports the tuner's timings of the layer alone
 * (fastest fused configuration, two-stage; -1 when not timed). */
int wino_batch_set_route(void* batch, int layer, int route);
int wino_batch_get_route(void* batch, int layer, int* route, float* fused_us, float* twostage_us);
int wino_batch_set_order(void* batch, const int* order, int n);
int wino_batch_get_order(void* batch, int* order, int n);
int wino_batch_commit(void* batch);
int wino_batch_run(void* batch, void* stream);
int wino_batch_tune(void* batch, int reps, float* layer_us, float* order_us, void* stream);
int wino_batch_graph_capture(void* batch, void* stream);
int wino_batch_graph_launch(void* batch, void* stream);

/* Launch the four slots of a kernelInfo_t filled by getkernelInfo, in order,
 * on `stream`, each with args[0] = param: the launch sequence of the
 * reference harness (reference src/main.cpp:105-108).  `ki` is `const
 * kernelInfo_t*` from conv2d.h, passed untyped so this header stands alone. */
int wino_launch_kernelinfo(const void* ki, void* param, void* stream);

/* Conv for callers that cannot allocate device memory (no counterpart in the
 * reference).  Plugin hosts that pass only input and output tensors, runtimes
 * whose device memory is fixed at start-up, and code that must not reach the
 * allocator mid-call cannot provide the U-cache workspace the other entry
 * points need; this one keeps U in a fixed array inside the library (8 MiB
 * held on every GPU that loads the library, for K*C <= wino_noalloc_max_kc())
 * and runs the filter transform and the fused conv on it.  Larger filters
 * return WINO_ESCRATCH.  Every call looks up the array's address on the
 * current device (nothing cached, so a cudaDeviceReset does not leave a stale
 * address); the first call on a device may also load the library's kernels,
 * so make it before any stream capture on that device.  All calls share the
 * array: calls whose kernels overlap on the GPU race, so serialise them.
 * Allocates nothing.  x: NCHW fp16, weight: KCRS fp16, y: N K H W fp16. */
int wino_conv2d_noalloc(const void* x, const void* weight, void* y, int n, int c, int h, int w,
                        int k, void* stream);
long long wino_noalloc_max_kc(void);

/* Self-test of the failure detection (no counterpart in the reference, which
 * has none): a kernel whose two bounded waits -- warp-wide and single-thread,
 * the forms the conv kernels use -- wait on mbarriers nothing signals, so
 * both run out after their time limit (~1 s), record their codes
 * (code[0] = 1, code[1] = 2 expected) and return normally.  Returns a
 * cudaError_t (0 = the kernel ended without a fault). */
int wino_selftest_wait_timeout(uint32_t* code);

/* Reads and clears the device error word of the conv kernels (0 = none;
 * otherwise the first wait that ran out or the first bad-shape launch). */
int wino_error_read_clear(uint32_t* code);

#ifdef __cplusplus
}
#endif

#endif /* WINO_WINOCONV_H */
