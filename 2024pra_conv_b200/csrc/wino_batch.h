// Layer table of the batched persistent launch, shared by the kernel
// (fused_conv.cu) and the host batch object (wino_batch.cpp).  Plain
// structs: the host builds a table and copies it to device memory once.
#pragma once
#include <cstdint>
#include "wino_param.h"

namespace wino {

// Schedule configuration bits of one layer.
//   CFG_KMAJOR  blocks ordered k-block-major (consecutive blocks share the U
//               k-block) instead of tile-major (they share input tiles);
//   CFG_DIRECT  producers read the NCHW input directly (no XB pre-pass).
constexpr int CFG_KMAJOR = 1, CFG_DIRECT = 2, NCFG = 4;

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
