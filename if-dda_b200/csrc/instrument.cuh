// Launch counting and optional CUDA-event timing of one mat-vec pass.
//
// Every kernel launch of the library goes through count_launch(); the bench
// reads the total to report how many of its own kernels ran.  When a pass is
// selected with ifdda_timing_enable(), the mat-vec launcher brackets each
// launch of that pass with a pair of CUDA events on the launching stream, so
// its average duration can be read after a timed region.
#pragma once
#include <cuda_runtime.h>
#include <atomic>

namespace ifdda {

enum MvPass { PASS_NONE = 0, PASS_FWD_X = 1, PASS_FWD_Y = 2, PASS_ZCONV = 3, PASS_INV_Y = 4, PASS_INV_X = 5 };

std::atomic<unsigned long long>& launch_counter();
inline void count_launch(unsigned n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

// returns the event to record before a launch of `pass` (or null when that
// pass is not being timed); timing_after() records the matching end event
cudaEvent_t timing_before(int pass, int precision_bytes, cudaStream_t st);
void timing_after(cudaEvent_t start, cudaStream_t st);
// true while a pass is selected for event timing
bool timing_active();

}  // namespace ifdda
