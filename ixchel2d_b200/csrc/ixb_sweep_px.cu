// Assembly of sweep EQ_PX in the reference's operation order (built without FMA contraction: bit-identical rows).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t assemble_launch<EQ_PX, IXB_SOLVER_EXACT>(const SweepShape&, const Geo<double>&,
                                                              const SweepIO<double>&, const StageBuf&, cudaStream_t);
template cudaError_t fused_launch<EQ_PX, IXB_SOLVER_EXACT>(const SweepShape&, const Geo<double>&, const SweepIO<double>&,
                                                   const SolveIO&, cudaStream_t);
}  // namespace ixb
