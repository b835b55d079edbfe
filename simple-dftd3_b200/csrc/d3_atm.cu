// Axilrod-Teller-Muto three-body kernels (placeholder until the triple kernel lands).
#include "d3_device.cuh"

namespace d3 {

void launch_three_body(const Batch&, const Species&, const Damp&, const Config&, const Partition&,
                       const Work&, long long, int, cudaStream_t)
{
}

}  // namespace d3
