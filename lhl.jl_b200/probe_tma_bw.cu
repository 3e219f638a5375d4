// probe_tma_bw.cu -- the streaming rate of the Hessenberg solve's TMA pipeline with no
// arithmetic: one producer warp requests 128 x 32 FP64 boxes of a Gt-shaped array (2052 rows)
// through a ring of 2..6 shared-memory slots, 16 consumer warps wait for each box and release
// it.  Prints the per-SM and total bandwidth for 1 CTA and for 64 CTAs (one per shift).
// This is the roofline of hess_tma_kernel: 1 CTA bounds one right-hand side, 64 CTAs a batch.
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -I include \
//        -o probe_tma_bw lhl.jl_b200/probe_tma_bw.cu -lcuda && ./probe_tma_bw
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include "csrc/common.cuh"
using namespace lhl;
constexpr int ROWS = 128, COLS = 32, NCONS = 16;
__device__ __forceinline__ void arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory"); }
__global__ void __launch_bounds__(544) k(int nbox, int ns, int colstride, const __grid_constant__ CUtensorMap tm, double* out) {
  extern __shared__ __align__(1024) double box[];
  __shared__ __align__(8) uint64_t full[8], empty[8];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) { for (int u = 0; u < ns; ++u) { mbar_init(&full[u], 1); mbar_init(&empty[u], NCONS); } mbar_fence_init(); }
  __syncthreads();
  const int col0 = blockIdx.x * colstride;
  if (warp == NCONS) {
    if (lane == 0) {
      for (int u = 0; u < nbox; ++u) {
        const int slot = u % ns;
        if (u >= ns) mbar_wait_ns(&empty[slot], (u / ns - 1) & 1, 2000000000ull);
        mbar_expect_tx(&full[slot], ROWS * COLS * 8);
        const int x = (u * ROWS) % 2048, y = col0 + ((u * ROWS) / 2048) * COLS % 2048;
        tma_load_2d(box + (size_t)slot * ROWS * COLS, &tm, x, y, &full[slot]);
      }
      for (int v = nbox > ns ? nbox - ns : 0; v < nbox; ++v) mbar_wait_ns(&full[v % ns], (v / ns) & 1, 2000000000ull);
    }
    return;
  }
  double acc = 0;
  for (int u = 0; u < nbox; ++u) {
    const int slot = u % ns;
    mbar_wait_ns(&full[slot], (u / ns) & 1, 2000000000ull);
    acc += box[(size_t)slot * ROWS * COLS + warp * ROWS + lane];
    __syncwarp();
    if (lane == 0) arrive(&empty[slot]);
  }
  if (acc == 12345.0) out[0] = acc;
}
int main() {
  const int ld = 2052, cols = 2048 * 64;
  double* G; cudaMalloc(&G, (size_t)ld * cols * 8); cudaMemset(G, 0, (size_t)ld * cols * 8);
  double* out; cudaMalloc(&out, 8);
  void* fn = nullptr; cudaDriverEntryPointQueryResult q;
  cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  CUtensorMap tm; cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)cols}; cuuint64_t str[1] = {(cuuint64_t)ld * 8};
  cuuint32_t boxd[2] = {ROWS, COLS}, es[2] = {1, 1};
  ((PFN_cuTensorMapEncodeTiled_v12000)fn)(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, G, dims, str, boxd, es,
     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  const int nbox = 544;
  for (int ns = 2; ns <= 6; ++ns) {
    const size_t sm = (size_t)ns * ROWS * COLS * 8;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    for (int grid : {1, 64}) {
      cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
      k<<<grid, 544, sm>>>(nbox, ns, 2048, tm, out);
      cudaEventRecord(a);
      for (int r = 0; r < 3; ++r) k<<<grid, 544, sm>>>(nbox, ns, 2048, tm, out);
      cudaEventRecord(b); cudaEventSynchronize(b);
      float ms; cudaEventElapsedTime(&ms, a, b); ms /= 3;
      const double bytes = (double)grid * nbox * ROWS * COLS * 8;
      printf("ns=%d grid=%d time=%.1f us  per-SM %.1f GB/s  total %.1f GB/s  err=%s\n", ns, grid, ms * 1e3,
             bytes / grid / (ms * 1e-3) / 1e9, bytes / (ms * 1e-3) / 1e9, cudaGetErrorString(cudaGetLastError()));
    }
  }
  return 0;
}
