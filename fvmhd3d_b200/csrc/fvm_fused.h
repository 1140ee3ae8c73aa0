// The persistent rung kernel's launch interface, shared by fvm_kernels.cu
// (which captures it into a partial step's graph) and fvm_fused.cu (which
// holds the kernel).  Included after fvm_device.cuh.
#pragma once

namespace fvm {

// Everything one partial step reads and writes, by value: the context's
// parameters and device arrays, the flux settings, and the grid barrier.
struct FusedStep {
  Params P;
  Dev d;
  LearnBuf lb;
  int n, nf;
  unsigned *gbar;  // grid barrier: arrivals (zero between launches), generation
  int *gerr;       // bit 1: a grid barrier wait gave up
};

// Enqueues one persistent launch of the partial step on `st`: every stage
// from the slope limiter to the reconstruction over the step's involved
// cells and active faces, with grid-wide barriers between the stages.  grid:
// fused_step_blocks_per_sm times the SM count.  Returns the CUDA error of the
// launch.
cudaError_t fused_step_enqueue(const FusedStep &a, bool fp32, int grid, cudaStream_t st);

// Blocks of the persistent kernel resident per SM (its grid is this times
// the SM count).
int fused_step_blocks_per_sm(bool fp32);

}  // namespace fvm
