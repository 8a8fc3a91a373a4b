#pragma once
// Read-bandwidth probe (probe.cu): the measured peaks behind the roofline figures.
#include <cstdint>

#include <cuda_runtime_api.h>

namespace rtg {

// Allocates a zero-filled buffer of `bytes` on the current device, reads it
// `reps` times per launch with 16-byte loads over a grid filling every SM, and
// reports the best of five launches in GB/s. l1 = false: loads bypass L1 and the
// grid shares the buffer (>= 1 MiB); well under the L2 size that measures L2
// read bandwidth, far above it HBM's. l1 = true: L1-cached loads, every block
// reads the whole buffer (4 KiB to 128 KiB): the aggregate L1 read bandwidth.
cudaError_t probe_read_bandwidth(std::uint64_t bytes, int reps, bool l1, cudaStream_t stream, double* gbs);

}  // namespace rtg
