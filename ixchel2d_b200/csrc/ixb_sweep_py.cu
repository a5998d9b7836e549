// Sweep kernel EQ_PY with the reference-order assembly and the sequential Thomas solve (bit-identical to the reference).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t sweep_launch_solver<double, EQ_PY, IXB_SOLVER_EXACT>(const SweepShape&, const Geo<double>&,
                                                                     const Geo<float>&, const SweepIO<double>&,
                                                                     cudaStream_t);
template cudaError_t sweep_smem_limit_solver<double, EQ_PY, IXB_SOLVER_EXACT>(int);
template int sweep_blocks_per_sm_solver<double, EQ_PY, IXB_SOLVER_EXACT>(const SweepShape&);
}  // namespace ixb
