// Mixed-precision instantiation of the batched step.
#include "i2g_batch.cuh"

namespace i2g {

int launch_batch_step_mixed(cudaStream_t s, const BatchRun &R, int move_ctas, int cell_ctas)
{
    return launch_batch_step_t<true>(s, R, move_ctas, cell_ctas);
}

}  // namespace i2g
