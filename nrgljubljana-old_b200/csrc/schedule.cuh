// Size-bucketed schedule of the batched step: the choices that depend on the
// device and are set by measurement (autotune.cu) rather than fixed in the
// code.  One table per device, shared by every context and server of the
// process; readers take the current values at each launch.
//
//   cluster_limit   blocks up to this size are tridiagonalised whole inside
//                   one thread-block cluster; larger ones take cooperative
//                   panel launches until their trailing block is this small
//                   (0: the cluster kernel's capacity, the default)
//   gemm_large_from grouped FP64 GEMM launches whose problems average at
//                   least this edge (sqrt of the output area) use 128 x 128
//                   tiles instead of 64 x 64 (0: never, the default)
#pragma once
#include <atomic>

namespace nrgb {

struct Schedule {
  std::atomic<int> cluster_limit{0};
  std::atomic<int> gemm_large_from{0};
  std::atomic<int> tuned{0};
};

// The table of `device` (0 <= device < 64).
Schedule& schedule_of(int device);
// The table of the current device.
Schedule& schedule_here();

}  // namespace nrgb
