// Assembly of sweep EQ_UX for the mixed-precision form (binary32 staged rows; built with FMA contraction).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t assemble_launch<EQ_UX, SOLVER_MIXED>(const SweepShape&, const Geo<double>&, const Geo<float>&,
                                                          const SweepIO<double>&, const StageBuf&, cudaStream_t);
}  // namespace ixb
