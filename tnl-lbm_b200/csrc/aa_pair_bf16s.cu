// Two-site step kernels (pair.cuh) for the bf16s population storage (StoreBF16S).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_bf16s, StoreBF16S)
