"""Throughput of global float reductions (RED) on this GPU: the ceiling of
the push / count / backward scatters -- a measurement script, not a test
(pytest does not collect it).

    python tests/perf_atomic_throughput.py

Compiles a small probe with nvcc (into a temporary folder) and runs it:
every thread issues 64 reductions into a 16 MB buffer (L2-resident), all
addresses in bounds and aligned for the vector forms.  Patterns: 32 lanes
on 32 consecutive floats; pairs / quads of lanes on one address; lanes two
floats apart; red.global.add.v2.f32 and .v4.f32 on consecutive vectors.
Prints warp-level reductions per second and float adds per second.
"""
import os
import subprocess
import sys
import tempfile

SOURCE = r"""
// Throughput probe of global float reductions on B200: scalar vs vector RED,
// distinct vs duplicate addresses within a warp.  All addresses in bounds.
#include <cstdio>
#include <cuda_runtime.h>
#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { printf("err %s line %d\n", cudaGetErrorString(e), __LINE__); return 1; } } while (0)

constexpr int K = 64;          // REDs per thread
constexpr int M = 1 << 22;     // floats in the buffer (16 MB)

// mode 0: scalar, lane -> base+lane; 1: scalar, lane -> base+lane/2 (pairs)
// 2: scalar, lane -> base+2*lane; 3: v2 at base+2*lane; 4: v4 at base+4*lane
// 5: scalar, lane -> base + lane/4 (quads)
template <int MODE>
__global__ void red_kernel(float* out) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int base = (warp * 97) & (M / 2 - 1);   // spread warps over the buffer
  base &= ~127;                           // 512-byte aligned
  for (int k = 0; k < K; ++k) {
    const int off = (base + k * 131 * 4) & (M / 2 - 1) & ~3;
    if (MODE == 0) atomicAdd(out + off + lane, 1.0f);
    if (MODE == 1) atomicAdd(out + off + lane / 2, 1.0f);
    if (MODE == 2) atomicAdd(out + off + 2 * lane, 1.0f);
    if (MODE == 5) atomicAdd(out + off + lane / 4, 1.0f);
    if (MODE == 3) {
      float* p = out + off + 2 * lane;
      asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" :: "l"(p), "f"(1.0f), "f"(1.0f) : "memory");
    }
    if (MODE == 4) {
      float* p = out + off + 4 * lane;
      asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" :: "l"(p), "f"(1.0f), "f"(1.0f), "f"(1.0f), "f"(1.0f) : "memory");
    }
  }
}

template <int MODE>
float run(float* out, int blocks) {
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  red_kernel<MODE><<<blocks, 256>>>(out);
  cudaEventRecord(a);
  for (int r = 0; r < 5; ++r) red_kernel<MODE><<<blocks, 256>>>(out);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms; cudaEventElapsedTime(&ms, a, b);
  return ms / 5;
}

int main() {
  float* out;
  // max offset: (M/2-1) + 4*31 + 3 < M
  CK(cudaMalloc(&out, sizeof(float) * M));
  CK(cudaMemset(out, 0, sizeof(float) * M));
  const int blocks = 148 * 8 * 16;
  const double reds = double(blocks) * 256 * K;   // thread-level RED instructions
  const double winst = reds / 32;
  float t;
  t = run<0>(out, blocks); printf("scalar distinct   : %.3f ms  %.1f G warp-RED/s  %.1f G lane-adds/s\n", t, winst / t / 1e6, reds / t / 1e6);
  t = run<1>(out, blocks); printf("scalar pairs dup  : %.3f ms  %.1f G warp-RED/s\n", t, winst / t / 1e6);
  t = run<5>(out, blocks); printf("scalar quads dup  : %.3f ms  %.1f G warp-RED/s\n", t, winst / t / 1e6);
  t = run<2>(out, blocks); printf("scalar stride2    : %.3f ms  %.1f G warp-RED/s\n", t, winst / t / 1e6);
  t = run<3>(out, blocks); printf("v2 (2 adds/lane)  : %.3f ms  %.1f G warp-RED/s  %.1f G lane-adds/s\n", t, winst / t / 1e6, 2 * reds / t / 1e6);
  t = run<4>(out, blocks); printf("v4 (4 adds/lane)  : %.3f ms  %.1f G warp-RED/s  %.1f G lane-adds/s\n", t, winst / t / 1e6, 4 * reds / t / 1e6);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  cudaFree(out);
  return 0;
}
"""


def main():
    with tempfile.TemporaryDirectory() as d:
        cu = os.path.join(d, "red_probe.cu")
        exe = os.path.join(d, "red_probe")
        with open(cu, "w") as f:
            f.write(SOURCE)
        subprocess.check_call(["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-o", exe, cu])
        sys.exit(subprocess.call([exe]))


if __name__ == "__main__":
    main()
