// cc_multi_launch.h — the fused multi-instance evaluation launch shared by the batch API and the server.
#pragma once
#include <cuda_runtime.h>

#include "cc_kernels.cuh"

namespace cc {

constexpr int kBatchChunk = 16;          // particles whose rho tables are built at once in a multi-instance launch
constexpr int kBatchPerSplit = 64;       // particles per rho block of an instance
constexpr int kBatchSegsPerSplit = 64;   // segments per force block of an instance

// One evaluation of B instances (any dimensions) in ONE launch of the fused batch kernel (cc_mbatch_kernel):
// mode 0 FP64, 1 mixed, 2 each instance at the precision of its stage word. rho_row / force_row: the largest table
// rows of the instances, maxd their largest dimension (they size the shared memory); the grid is the kernel's resident
// blocks (or fewer when there are fewer items).
int launch_mbatch(int mode, const MBatchArgs &a, int rho_row, int force_row, int maxd, cudaStream_t st);

}  // namespace cc
