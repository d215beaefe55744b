// rmat.cu -- device RMAT edge generator, bit-exact with the reference's
// rMat<uint32_t> (include/rmat_util.h:81-115): edge i walks log2(n) levels;
// level j draws r = hash32(start + j*stride) / INT32_MAX (so r lies in
// [0,2) and the quadrant probabilities are a/2, b/2, c/2, rest), with
// start = hash32(2i*h), stride = hash32((2i+1)*h), h = hash32(seed).
#include "trc_common.cuh"

namespace trc {

__device__ __forceinline__ uint32_t dev_hash32(uint32_t a) {
  a = (a + 0x7ed55d16u) + (a << 12);
  a = (a ^ 0xc761c23cu) ^ (a >> 19);
  a = (a + 0x165667b1u) + (a << 5);
  a = (a + 0xd3a2646cu) ^ (a << 9);
  a = (a + 0xfd7046c5u) + (a << 3);
  a = (a ^ 0xb55a4f09u) ^ (a >> 16);
  return a;
}

__global__ void k_rmat(uint32_t n, uint32_t h, double a, double ab, double abc, uint64_t first,
                       uint64_t count, uint32_t *src, uint32_t *dst) {
  uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  uint32_t i = (uint32_t)(first + k);
  uint32_t rs = dev_hash32((2u * i) * h);
  uint32_t st = dev_hash32((2u * i + 1u) * h);
  uint32_t x = 0, y = 0;
  for (uint32_t nn = n; nn > 1; nn >>= 1) {
    double r = (double)dev_hash32(rs) / 2147483647.0;
    uint32_t half = nn >> 1;
    if (r < a) {
    } else if (r < ab) {
      y += half;
    } else if (r < abc) {
      x += half;
    } else {
      x += half;
      y += half;
    }
    rs += st;
  }
  src[k] = x;
  dst[k] = y;
}

void rmat_generate(uint32_t n, uint32_t seed, double a, double b, double c, uint64_t first,
                   uint64_t count, uint32_t *src, uint32_t *dst, cudaStream_t s) {
  uint32_t h = 0;
  {
    uint32_t x = seed;
    x = (x + 0x7ed55d16u) + (x << 12);
    x = (x ^ 0xc761c23cu) ^ (x >> 19);
    x = (x + 0x165667b1u) + (x << 5);
    x = (x + 0xd3a2646cu) ^ (x << 9);
    x = (x + 0xfd7046c5u) + (x << 3);
    x = (x ^ 0xb55a4f09u) ^ (x >> 16);
    h = x;
  }
  uint64_t blocks = ceil_div(count, 256);
  if (blocks) k_rmat<<<(unsigned)blocks, 256, 0, s>>>(n, h, a, a + b, a + b + c, first, count, src, dst);
  TRC_CUDA(cudaGetLastError());
}

}  // namespace trc
