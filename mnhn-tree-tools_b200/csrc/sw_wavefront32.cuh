// 32-bit warp wavefront over one pair, shared by the explicit-pair kernels.
#pragma once
#include <cstdint>

#include "sw_kernels.cuh"

namespace swgpu {

// ---------------------------------------------------------------------------
// Generic 32-bit warp wavefront (one pair per warp, 512-column chunks).
// ---------------------------------------------------------------------------
// Returns max H of the pair.  A (rows) may be any length; B (columns) is
// processed in 512-column chunks, lane 31 handing the chunk's last column to
// the next chunk through scratch[0..la) (written before it is read, so the
// scratch needs no clearing).
static __device__ int sw32_warp(const uint8_t* __restrict__ A, int la, const uint8_t* __restrict__ B, int lb,
                         int* __restrict__ scratch, int lane) {
  int mx = 0;
  const int nchunks = lb > 0 ? (lb + GEN_CHUNK - 1) / GEN_CHUNK : 0;
  for (int c = 0; c < nchunks; ++c) {
    const int c0 = c * GEN_CHUNK;
    int bc[GEN_W], H[GEN_W];
#pragma unroll
    for (int k = 0; k < GEN_W; ++k) {
      const int col = c0 + lane * GEN_W + k;
      bc[k] = col < lb ? (int)B[col] : 0x1FF;  // never equal to a row code
      H[k] = 0;
    }
    const bool first = (c == 0), lastchunk = (c == nchunks - 1);
    int last = 0, diag = 0;
    for (int s = 0; s < la + 32; ++s) {
      int left = __shfl_up_sync(0xFFFFFFFFu, last, 1);
      const int r = s - lane;
      const bool live = (r >= 0 && r < la);
      if (lane == 0) left = (first || !live) ? 0 : scratch[r];
      const int a = live ? (int)A[r] : 0x2FF;
      int hd = diag;
      int x = __vimax_s32_relu(left, H[0]);
#pragma unroll
      for (int k = 0; k < GEN_W; ++k) {
        const int d = (a == bc[k]) ? 7 : -1;
        const int v = __viaddmax_s32(hd, d, x);
        const int h = __viaddmax_s32_relu(v, -3, 0);
        if (k + 1 < GEN_W) x = __viaddmax_s32_relu(v, -3, H[k + 1]);
        hd = H[k];
        H[k] = h;
        mx = max(mx, h);
      }
      last = H[GEN_W - 1];
      if (lane == 31 && !lastchunk && live) scratch[r] = last;
      diag = left;
    }
    __syncwarp();
  }
  return __reduce_max_sync(0xFFFFFFFFu, mx);
}

}  // namespace swgpu
