// Instantiation of the fused sweep kernel for EQ_TX (one translation unit per sweep).
#include "ixb_sweep.cuh"

namespace ixb {
template cudaError_t sweep_launch<double, EQ_TX>(int, const SweepShape&, const Geo<double>&, const SweepIO<double>&,
                                                     cudaStream_t);
template cudaError_t sweep_smem_limit<double, EQ_TX>(int);
template int sweep_blocks_per_sm<double, EQ_TX>(int, const SweepShape&);
}  // namespace ixb
