// Sweep kernel EQ_UY of the mixed-precision solver (binary32 line solve on binary64 fields; built with FMA contraction).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t sweep_launch_solver<double, EQ_UY, SOLVER_MIXED>(const SweepShape&, const Geo<double>&,
                                                                   const Geo<float>&, const SweepIO<double>&,
                                                                   cudaStream_t);
template cudaError_t sweep_smem_limit_solver<double, EQ_UY, SOLVER_MIXED>(int);
template int sweep_blocks_per_sm_solver<double, EQ_UY, SOLVER_MIXED>(const SweepShape&);
}  // namespace ixb
