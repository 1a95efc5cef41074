// Optional CUDA-event timing of selected kernel launches (on the stream each
// kernel is launched on), with the algorithmic work of every launch, for the
// roofline numbers of the benchmark.  Off unless aosb_kernel_timing(1).
#pragma once

#include "common.cuh"

namespace aosb {

enum TimedKernel : int {
  kTimedSchur = 0,        // schur_tc_kernel, Schur items
  kTimedSolveDiag = 1,    // solve_diag_kernel
  kTimedSolveUpdate = 2,  // solve_update_kernel / solve_tc_kernel
  kTimedResidual = 3,     // shifted_residual(_blocks)_kernel
  kTimedSpmm = 4,         // spmm_kernel
  kTimedBloch = 5,        // bloch_windows_kernel
  kTimedCount = 6,
};

// Records a start event on `st` and returns true when timing is on (and the
// stream is not being captured).
bool timing_begin(cudaStream_t st, cudaEvent_t (&ev)[2]);
// Records the stop event and books the launch under `cat`.
void timing_end(int cat, cudaStream_t st, cudaEvent_t (&ev)[2], double flops, double bytes);

}  // namespace aosb
