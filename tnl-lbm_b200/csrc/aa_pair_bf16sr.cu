// Two-site step kernels (pair.cuh) for the bf16sr population storage (StoreBF16SR).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_bf16sr, StoreBF16SR)
