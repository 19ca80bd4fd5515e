// Two-site step kernels (pair.cuh) for the f16sr population storage (StoreF16SR).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_f16sr, StoreF16SR)
