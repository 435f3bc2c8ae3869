// Persistent tile-task kernel for many small FP64 reconstructor instances
// (packed.cu).
#ifndef MOAO_PACKED_H
#define MOAO_PACKED_H

#include <vector>

#include "context.h"

namespace moao {

// One instance: Cmm (n x n, lower, lda) is factored in place; C holds Ctm
// (m x n, ldc) and ends as R = Ctm Cmm^-1; info (device) receives the first
// failing Cholesky column (1-based) and must be zeroed by the caller.
struct PackedInst {
  double* A = nullptr;
  long lda = 0;
  double* C = nullptr;
  long ldc = 0;
  long n = 0, m = 0;
  int* info = nullptr;
};

// Device state of one packed launch: instance table, level-sorted task list,
// tile counters, inverse diagonal tiles, claim counter and error flag.
struct PackedPlan {
  DevBuf inst, tasks, cnt, linv, ctl;
  long ntasks = 0;
  int levels = 0;
  size_t cnt_bytes = 0;
  void release();
};

// Device bytes of the plan's per-instance state (inverse tiles, counters, tasks).
size_t packed_workspace_bytes(long n, long m);
// Builds and uploads the task list (host work, synchronous on s; not capturable).
moao_status packed_prepare(const std::vector<PackedInst>& v, PackedPlan* plan, cudaStream_t s);
// Resets the counters and launches the persistent kernel on s (capturable).
// polls > 0 bounds every dependency wait to that many polls; wait_s bounds it in
// time. On expiry the kernel stops and *packed_error_flag(plan) is nonzero.
moao_status packed_launch(const PackedPlan& plan, cudaStream_t s, unsigned long long polls,
                          double wait_s, long long* launches);
const int* packed_error_flag(const PackedPlan& plan);

}  // namespace moao

#endif  // MOAO_PACKED_H
