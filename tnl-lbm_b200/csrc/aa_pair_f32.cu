// Two-site step kernels (pair.cuh) for the f32 population storage (StoreF32).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_f32, StoreF32)
