// Two-site step kernels (pair.cuh) for the i16s population storage (StoreI16S).
#include "pair.cuh"

LBM_DEFINE_PAIR_STEP(pair_step_i16s, StoreI16S)
