// fr_peaks.cu -- measured roofs of the scattered accumulation that bounds
// the insertion kernels.  The insertion is not a dense contraction and its
// compulsory HBM bytes are tiny next to its taps (a gauss_5 tap adds three
// floats to a voxel), so beside the HBM copy bandwidth the binding roof is
// the rate at which the device can apply those adds.  Three forms:
//   smem_rmw : conflict-free float4 read-modify-write in shared memory (the
//              column kernel's owner-computes accumulator update, one per tap)
//   smem_atom: FP32 atomicAdd to random shared-memory words (3 per tap)
//   l2_red   : FP32 red.global.add to random words of an L2-resident buffer
//              (the scatter schedule's update, 3 per tap)
// Each is timed with CUDA events on a private stream after one warm-up launch.
#include <cuda_runtime.h>

#include <cstdint>

#include "fr_handle.h"

namespace fr {
namespace {

constexpr int kRmwSlots = 1024;  // float4 per CTA (16 KB): 8 CTAs per SM fit

__global__ void __launch_bounds__(256) k_smem_rmw(float *out, int iters) {
  __shared__ float4 acc[kRmwSlots];
  for (int i = threadIdx.x; i < kRmwSlots; i += blockDim.x) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  const float a = 1.0f + threadIdx.x * 1e-3f;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(acc);
  for (int it = 0; it < iters; it++) {
    // consecutive lanes touch consecutive float4 slots: no bank conflicts.
    // Volatile shared accesses, so every update is a real load and store.
    const uint32_t addr = base + 16u * ((it * 256 + threadIdx.x) & (kRmwSlots - 1));
    float x, y, z, w;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(x), "=f"(y), "=f"(z), "=f"(w) : "r"(addr) : "memory");
    x += a;
    y -= a;
    z += 0.5f * a;
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "r"(addr), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
  }
  __syncthreads();
  float t = 0.f;
  for (int i = threadIdx.x; i < kRmwSlots; i += blockDim.x) t += acc[i].x + acc[i].y + acc[i].z;
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

constexpr int kAtomWords = 12288;  // 48 KB per CTA

__global__ void __launch_bounds__(256) k_smem_atom(float *out, int iters) {
  __shared__ float acc[kAtomWords];
  for (int i = threadIdx.x; i < kAtomWords; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  uint32_t s = threadIdx.x * 2654435761u + blockIdx.x * 97u + 1u;
  for (int it = 0; it < iters; it++) {
    s = s * 1664525u + 1013904223u;
    const int idx = (int)((s >> 8) % (uint32_t)(kAtomWords - 2));
    atomicAdd(&acc[idx], 1.0f);
    atomicAdd(&acc[idx + 1], 0.5f);
    atomicAdd(&acc[idx + 2], 0.25f);
  }
  __syncthreads();
  float t = 0.f;
  for (int i = threadIdx.x; i < kAtomWords; i += blockDim.x) t += acc[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = t;
}

__global__ void __launch_bounds__(256) k_l2_red(float *buf, uint32_t words, int iters) {
  uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 7u;
  for (int it = 0; it < iters; it++) {
    s = s * 1664525u + 1013904223u;
    const uint32_t idx = (s >> 4) % (words - 2);
    atomicAdd(&buf[idx], 1.0f);
    atomicAdd(&buf[idx + 1], 0.5f);
    atomicAdd(&buf[idx + 2], 0.25f);
  }
}

}  // namespace
}  // namespace fr

using namespace fr;

extern "C" FR_API int fr_update_peaks(double *smem_rmw_taps, double *smem_atom_taps,
                                      double *l2_red_taps) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return fail(FR_ECUDA, "fr_update_peaks: no CUDA device");
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float *out = nullptr, *buf = nullptr;
  const int grid_rmw = sms * 8, grid_atom = sms * 4, grid_red = sms * 8;
  const uint32_t red_words = 4u << 20;  // 16 MB: resident in L2
  const size_t nout = (size_t)grid_rmw * 256;
  int rc = FR_OK;
  auto run = [&](int which, int iters, double per_thread_taps, int grid, double *res) -> bool {
    float ms = 0.f;
    for (int rep = 0; rep < 2; rep++) {
      if (cudaEventRecord(e0, st) != cudaSuccess) return false;
      if (which == 0) k_smem_rmw<<<grid, 256, 0, st>>>(out, iters);
      else if (which == 1) k_smem_atom<<<grid, 256, 0, st>>>(out, iters);
      else k_l2_red<<<grid, 256, 0, st>>>(buf, red_words, iters);
      if (cudaGetLastError() != cudaSuccess) return false;
      if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
        return false;
      if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return false;
    }
    if (res) *res = (double)grid * 256.0 * per_thread_taps / (ms * 1e-3);
    return true;
  };
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
      cudaMalloc(&out, nout * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&buf, (size_t)red_words * sizeof(float)) != cudaSuccess ||
      cudaMemsetAsync(buf, 0, (size_t)red_words * sizeof(float), st) != cudaSuccess) {
    rc = fail(FR_ECUDA, "fr_update_peaks: setup failed");
  } else if (!run(0, 8192, 8192.0, grid_rmw, smem_rmw_taps) ||
             !run(1, 2048, 2048.0, grid_atom, smem_atom_taps) ||
             !run(2, 1024, 1024.0, grid_red, l2_red_taps)) {
    rc = fail(FR_ECUDA, "fr_update_peaks: kernel failed");
  }
  if (out) cudaFree(out);
  if (buf) cudaFree(buf);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  return rc;
}
