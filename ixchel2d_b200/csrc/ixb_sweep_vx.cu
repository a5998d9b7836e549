// Instantiation of the fused sweep kernel for EQ_VX (one translation unit per sweep).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t sweep_launch<double, EQ_VX>(int, const SweepShape&, const Geo<double>&, const SweepIO<double>&,
                                                     cudaStream_t);
template cudaError_t sweep_smem_limit<double, EQ_VX>(int);
template int sweep_blocks_per_sm<double, EQ_VX>(int, const SweepShape&);
}  // namespace ixb
