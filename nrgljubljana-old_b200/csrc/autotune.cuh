// Autotuner of the size-bucketed schedule (schedule.cuh): measures on the
// current device and sets its table; returns a JSON report of what it timed
// and chose.  Runs its own synthetic work on `st` (a few seconds).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>

#include "syev.cuh"

namespace nrgb {

std::string autotune(EigSolver& syev, int cluster_capacity, cudaStream_t st);

}  // namespace nrgb
