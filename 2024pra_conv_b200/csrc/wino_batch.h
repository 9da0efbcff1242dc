// Layer table of the batched persistent launch, shared by the kernel
// (fused_conv.cu) and the host batch object (wino_batch.cpp).  Plain
// structs: the host builds a table and copies it to device memory once.
#pragma once
#include <cstdint>
#include "wino_param.h"

namespace wino {

// Schedule configuration of one layer (bits):
//   CFG_KMAJOR  blocks ordered k-block-major (consecutive blocks share the U
//               k-block) instead of tile-major (they share input tiles);
//   CFG_DIRECT  producers read the NCHW input directly (no XB pre-pass);
//   bits 2-3    split level L: the 16-channel steps of each (tile block,
//               k block) are split over up to 4^L CTAs, which add fp32 partial
//               outputs into a buffer (p.mid_result) that a second pass
//               rounds to fp16 -- for layers with too few blocks to fill the
//               GPU.  Single-layer fp16 launches only.
constexpr int CFG_KMAJOR = 1, CFG_DIRECT = 2, CFG_SPLIT_SHIFT = 2, NCFG = 16;

__host__ __device__ inline int cfg_split_level(int cfg) { return (cfg >> CFG_SPLIT_SHIFT) & 3; }

// Splits actually used for `cs` steps: every split non-empty.
__host__ __device__ inline void split_plan(int cfg, int cs, int& nsplit, int& per) {
  const int want = 1 << (2 * cfg_split_level(cfg));
  per = (cs + want - 1) / want;
  if (per < 1) per = 1;
  nsplit = (cs + per - 1) / per;
}

constexpr int BATCH_MAX = 32;  // layers per table

struct LayerDesc {
  KernelParam p;            // pin, pout, transform_pin (XB), transform_filter (U)
  long long block_begin;    // first global block of the layer
  int cfg;
  int pad;
};

struct BatchTable {
  int nlayers, pad;
  long long total;
  LayerDesc layer[BATCH_MAX];
};

}  // namespace wino
