// cc_multi_launch.h — the multi-instance evaluation launch shared by the batch API and the server.
#pragma once
#include <cuda_runtime.h>

#include "cc_kernels.cuh"

namespace cc {

constexpr int kBatchChunk = 16;          // particles whose rho tables are built at once in a multi-instance launch
constexpr int kBatchPerSplit = 64;       // particles per rho block of an instance
constexpr int kBatchSegsPerSplit = 64;   // segments per force block of an instance

// One evaluation of B instances of dimension D: the persistent rho, reduce and force kernels (programmatic
// dependent launch) over per-instance arguments on the device. pre: 3 x (B + 1) prefix sums of the instances' blocks
// (rho, reduce, force), shape: 3 x B (block groups, reduce chunks, particle groups), total: the three sums;
// rho_row / force_row: the largest table rows; queue: 6 zeroed words (reset by the kernels). MIXED for the mixed
// precision kernels; instances whose stage word differs from 0 (mixed) or 1 (FP64) are skipped.
int launch_multi(int D, bool mixed, const RhoArgs *rho, const ReduceArgs *red, const ForceArgs *force, const int *pre,
                 const int *shape, int B, const int total[3], int rho_row, int force_row, unsigned *queue,
                 cudaStream_t st);

}  // namespace cc
