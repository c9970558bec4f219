// FP64 instantiation of the batched step (built with --fmad=false, like i2g_fp64.cu).
#include "i2g_batch.cuh"

namespace i2g {

int launch_batch_step_fp64(cudaStream_t s, const BatchRun &R, int move_ctas, int cell_ctas)
{
    return launch_batch_step_t<false>(s, R, move_ctas, cell_ctas);
}

int avg_smem_bytes(bool mixed) { return mixed ? (int)sizeof(AvgSmem<true>) : (int)sizeof(AvgSmem<false>); }

}  // namespace i2g
