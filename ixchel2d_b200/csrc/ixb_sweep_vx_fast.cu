// Assembly of sweep EQ_VX in the fast binary64 form (reciprocal tables; built with FMA contraction).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t assemble_launch<EQ_VX, IXB_SOLVER_HYBRID>(const SweepShape&, const Geo<double>&,
                                                               const SweepIO<double>&, const StageBuf&, cudaStream_t);
template cudaError_t assemble_batch_launch<EQ_VX, IXB_SOLVER_HYBRID>(const void*, const int2*, int, const int*, const BatchNorm&,
                                                           cudaStream_t);
template cudaError_t fused_launch<EQ_VX, IXB_SOLVER_HYBRID>(const SweepShape&, const Geo<double>&, const SweepIO<double>&,
                                                   const SolveIO&, cudaStream_t);
template cudaError_t fused_batch_launch<EQ_VX, IXB_SOLVER_HYBRID>(int, int, size_t, const FusedInst*, const int2*, int, const int*,
                                                         const BatchNorm&, const BatchNorm&, cudaStream_t);
}  // namespace ixb
