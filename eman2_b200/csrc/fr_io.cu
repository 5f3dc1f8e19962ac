// fr_io.cu -- decoding of raw particle-stack bytes on the device.  Image
// files are read as raw bytes into pinned host memory and copied to HBM
// undecoded (a 16-bit stack moves half the bytes of its float32 image); one
// pass widens them to float32 here, the way MrcIO::read_data converts each
// mode on the host (libEM/io/mrcio.cpp:1040-1140).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fr_handle.h"

namespace fr {
namespace {

__device__ __forceinline__ uint16_t swap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }
__device__ __forceinline__ uint32_t swap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

// mode: MRC mode number; swap: the file's byte order differs from the host's.
__global__ void k_decode(const unsigned char *__restrict__ src, int mode, int swap, long n,
                         float *__restrict__ dst) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = 0.0f;
  switch (mode) {
    case 0:    // MRC_UCHAR: unsigned bytes
      v = (float)src[i];
      break;
    case 17:   // MRC_CHAR: signed bytes
      v = (float)(signed char)src[i];
      break;
    case 101: {  // MRC_UHEX: two 4-bit values per byte, low nibble first
      const unsigned int b = src[i >> 1];
      v = (float)((i & 1) ? (b >> 4) : (b & 15));
      break;
    }
    case 1: {  // MRC_SHORT
      uint16_t u = reinterpret_cast<const uint16_t *>(src)[i];
      if (swap) u = swap16(u);
      v = (float)(int16_t)u;
      break;
    }
    case 6: {  // MRC_USHORT
      uint16_t u = reinterpret_cast<const uint16_t *>(src)[i];
      if (swap) u = swap16(u);
      v = (float)u;
      break;
    }
    case 12: {  // MRC_FLOAT16
      uint16_t u = reinterpret_cast<const uint16_t *>(src)[i];
      if (swap) u = swap16(u);
      v = __half2float(__ushort_as_half(u));
      break;
    }
    default: {  // 2, MRC_FLOAT
      uint32_t u = reinterpret_cast<const uint32_t *>(src)[i];
      if (swap) u = swap32(u);
      v = __uint_as_float(u);
      break;
    }
  }
  dst[i] = v;
}

}  // namespace
}  // namespace fr

using namespace fr;

extern "C" FR_API int fr_decode_images(const void *d_src, int mode, int swap, long long n,
                                       float *d_dst, void *stream) {
  if (!d_src || !d_dst) return fail(FR_ENULL, "null buffer");
  if (mode != 0 && mode != 1 && mode != 2 && mode != 6 && mode != 12 && mode != 17 && mode != 101)
    return fail(FR_EUNSUPPORTED, "MRC mode %d is not decoded", mode);
  if (!is_device_ptr(d_src) || !is_device_ptr(d_dst))
    return fail(FR_EINVAL_PARAM, "fr_decode_images takes device buffers");
  if (n <= 0) return FR_OK;
  note_launch();
  k_decode<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      (const unsigned char *)d_src, mode, swap ? 1 : 0, (long)n, d_dst);
  CU(cudaGetLastError());
  return FR_OK;
}
