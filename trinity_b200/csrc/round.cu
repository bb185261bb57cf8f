/*
 * round.cu — the end of a coarsening or swapping level, on the device.
 *
 * A free-mode level reads the list of active entities in one buffer and
 * appends the ones it re-activates to another. k_level_end moves the new list
 * into the first buffer (so every level runs the same kernels on the same
 * buffers), accumulates the call's statistics, bounds the number of levels,
 * advances the seed counter, and decides whether another level runs: for a
 * coarsening level, while it found candidates and collapsed some (the loop of
 * Coarse::run, coarsening.cpp:480-503); for a swapping level, while it flipped
 * some (Swap::run, swapping.cpp:395-425). The host-driven loop reads that
 * decision back; a captured round hands it to the loop node.
 */
#include "trn_internal.h"

namespace trn {

__global__ void k_level_end(int* status, int kind, int cap, const int* __restrict__ next,
                            int* __restrict__ cur, cudaGraphConditionalHandle h, int use_h) {
  const int n = status[S_ACT + 1];
  for (int i = trn_tid(); i < n; i += trn_grid_stride()) cur[i] = next[i];
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  level_end_decide(status, kind, cap, h, use_h);
}

void level_end(int* status, int kind, int cap, const int* next, int* cur, int hint, cudaStream_t s,
               cudaGraphConditionalHandle h, bool use_h) {
  k_level_end<<<grid_for(hint), TRN_THREADS, 0, s>>>(status, kind, cap, next, cur, h, use_h ? 1 : 0);
  note_launch();
  check_launch("level_end");
}

}  // namespace trn
