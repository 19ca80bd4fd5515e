// Two-site step kernels (pair.cuh) for the f16s population storage (StoreF16S).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_f16s, StoreF16S)
