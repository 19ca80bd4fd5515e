// Two-site step kernels (pair.cuh) for the f32s population storage (StoreF32S).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_f32s, StoreF32S)
