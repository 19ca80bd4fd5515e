// Two-site coupled flow + D3Q7 scalar step (ade_pair.cuh) for the f32 population storage.
#include "ade_pair.cuh"

namespace lbm {
cudaError_t ade_pair_step_f32(const StepLaunch& L)
{
	return ade_pair_step<StoreF32>(L);
}
}  // namespace lbm
