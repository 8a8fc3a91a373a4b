#pragma once
// Process-wide count of the memory allocations this library asks CUDA for
// (device, stream-ordered pool and pinned host). A diagnostic: it lets a caller
// check that an entry point which promises not to allocate really does not.
#include <cstdint>

namespace rtg {

void count_allocation();
std::uint64_t allocation_count();

}  // namespace rtg
