// 3xTF32 split-precision products on the tensor cores (mma.sync m16n8k8,
// FP32 accumulation), the mixed-precision form of the element contractions.
//
// A value x is held as the pair hi = tf32(x), lo = tf32(x - hi) (round to
// nearest, ties away, at the 10-bit TF32 mantissa): hi + lo carries about 21
// significant bits.  A product a b is accumulated as a_lo b_hi + a_hi b_lo +
// a_hi b_hi; the dropped a_lo b_lo term is below 2^-21 relative, so with FP32
// accumulation a k-term sum is good to a few FP32 ulps of its terms' magnitude.
// Operands are stored as uint2 {hi, lo} bit patterns in the 8 bytes a double
// would take, so FP64 and split layouts share one indexing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hfem {

__device__ __forceinline__ uint32_t tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ uint2 tf32_split(double x) {
    const uint32_t hi = tf32_rna((float)x);
    const uint32_t lo = tf32_rna((float)(x - (double)__uint_as_float(hi)));
    return make_uint2(hi, lo);
}

// c (16 x 8, FP32) += A (16 x 8) B (8 x 8), TF32 operands:
// a0 = A(g, t), a1 = A(g + 8, t), a2 = A(g, t + 4), a3 = A(g + 8, t + 4),
// b0 = B(t, g), b1 = B(t + 4, g), c = C(g, 2t .. 2t+1), C(g + 8, 2t .. 2t+1)
// with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// c += A B with A = ah + al and B = (b0, b1) as {hi, lo} pairs.
__device__ __forceinline__ void mma_3xtf32(float (&c)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4], uint2 b0,
                                           uint2 b1) {
    mma_tf32(c, al[0], al[1], al[2], al[3], b0.x, b1.x);
    mma_tf32(c, ah[0], ah[1], ah[2], ah[3], b0.y, b1.y);
    mma_tf32(c, ah[0], ah[1], ah[2], ah[3], b0.x, b1.x);
}

// A B-operand or Y entry: the double itself, or its {hi, lo} split.
template <bool TF>
__device__ __forceinline__ void bput(double* p, double v) {
    if constexpr (TF)
        *reinterpret_cast<uint2*>(p) = tf32_split(v);
    else
        *p = v;
}

}  // namespace hfem
