// Warp-level tensor-core products (mma.sync m16n8k8 with TF32 operands and
// FP32 accumulation) with the operands split into a TF32 head and tail, so
// that a product of FP32 numbers keeps about FP32 accuracy:
//   a = hi(a) + lo(a) + O(2^-22 |a|),   hi, lo TF32 (round to nearest),
//   a b ~ hi(a) hi(b) + hi(a) lo(b) + lo(a) hi(b)   (lo lo dropped, 2^-22).
// Fragment layout of m16n8k8 (lane = 4 g + t, g = 0..7, t = 0..3):
//   A (16 x 8, row-major): a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4]
//   B (8 x 8, column-major): b0 = B[t][g], b1 = B[t+4][g]
//   C (16 x 8): c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1]
#pragma once
#include <cstdint>

namespace qcd {

// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away
// from zero: half a TF32 unit in the last place added to the magnitude bits,
// the 13 bits below the TF32 mantissa cleared (a carry out of the mantissa
// steps the exponent, as rounding up must)
__device__ __forceinline__ uint32_t tf32_rn(float x) { return (__float_as_uint(x) + 0x1000u) & 0xffffe000u; }

// x = hi + lo with hi, lo TF32
struct Tf32x2 {
  uint32_t hi, lo;
};
__device__ __forceinline__ Tf32x2 tf32_split(float x) {
  Tf32x2 s;
  s.hi = tf32_rn(x);
  s.lo = tf32_rn(x - __uint_as_float(s.hi));
  return s;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// c += A B with A, B given as head/tail pairs (three tensor-core products,
// the small ones first)
__device__ __forceinline__ void mma_tf32x3(float (&c)[4], const Tf32x2 (&a)[4], const Tf32x2 (&b)[2]) {
  mma_tf32(c, a[0].lo, a[1].lo, a[2].lo, a[3].lo, b[0].hi, b[1].hi);
  mma_tf32(c, a[0].hi, a[1].hi, a[2].hi, a[3].hi, b[0].lo, b[1].lo);
  mma_tf32(c, a[0].hi, a[1].hi, a[2].hi, a[3].hi, b[0].hi, b[1].hi);
}

// acc += A B as above, the three products summed on the tensor cores from
// zero and then added to acc in FP32 with round-to-nearest.  The tensor
// cores' own additions are not round-to-nearest (they align the terms to the
// largest exponent and drop the bits below; Fasi, Higham, Mikaitis and
// Pranesh, "Numerical behavior of NVIDIA tensor cores", PeerJ Comput. Sci.
// 7:e330, 2021), so a long chain of products into one accumulator would
// pile up a one-sided error.
__device__ __forceinline__ void mma_tf32x3_add(float (&acc)[4], const Tf32x2 (&a)[4], const Tf32x2 (&b)[2]) {
  float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  mma_tf32x3(d, a, b);
#pragma unroll
  for (int i = 0; i < 4; i++) acc[i] += d[i];
}

}  // namespace qcd
