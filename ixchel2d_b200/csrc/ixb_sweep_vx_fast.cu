// Sweep kernel EQ_VX with the fast assembly and the partitioned Thomas-PCR solve (built with FMA contraction).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t sweep_launch_solver<double, EQ_VX, IXB_SOLVER_HYBRID>(const SweepShape&, const Geo<double>&,
                                                                     const Geo<float>&, const SweepIO<double>&,
                                                                     cudaStream_t);
template cudaError_t sweep_smem_limit_solver<double, EQ_VX, IXB_SOLVER_HYBRID>(int);
template int sweep_blocks_per_sm_solver<double, EQ_VX, IXB_SOLVER_HYBRID>(const SweepShape&);
}  // namespace ixb
