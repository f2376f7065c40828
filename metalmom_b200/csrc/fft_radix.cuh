// Register-resident DFT butterflies (forward, W = exp(-2*pi*i/R)) used by the
// Stockham stages of the frame FFT.  All arithmetic is float32; the constant
// twiddles below are cos/sin of multiples of pi/8, written out to 20 digits.
#pragma once
#include <cuda_runtime.h>

namespace mm {

struct cpx {
  float x, y;
};

__device__ __forceinline__ cpx cadd(cpx a, cpx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cpx csub(cpx a, cpx b) { return {a.x - b.x, a.y - b.y}; }
// a * b
__device__ __forceinline__ cpx cmul(cpx a, cpx b) {
  return {fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)};
}
// a * (-i)
__device__ __forceinline__ cpx mul_mi(cpx a) { return {a.y, -a.x}; }
// a * (+i)
__device__ __forceinline__ cpx mul_pi(cpx a) { return {-a.y, a.x}; }

constexpr float kR = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC1 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS1 = 0.38268343236508977173f;  // sin(pi/8)

// a * exp(-i*pi/4) = a * (R - iR)
__device__ __forceinline__ cpx mul_w8_1(cpx a) { return {kR * (a.x + a.y), kR * (a.y - a.x)}; }
// a * exp(-3i*pi/4) = a * (-R - iR)
__device__ __forceinline__ cpx mul_w8_3(cpx a) { return {kR * (a.y - a.x), -kR * (a.x + a.y)}; }
// a * exp(-i*pi/8) = a * (C1 - i S1)
__device__ __forceinline__ cpx mul_w16_1(cpx a) {
  return {fmaf(a.x, kC1, a.y * kS1), fmaf(a.y, kC1, -a.x * kS1)};
}
// a * exp(-3i*pi/8) = a * (S1 - i C1)
__device__ __forceinline__ cpx mul_w16_3(cpx a) {
  return {fmaf(a.x, kS1, a.y * kC1), fmaf(a.y, kS1, -a.x * kC1)};
}
// a * exp(-9i*pi/8) = -(a * exp(-i*pi/8))
__device__ __forceinline__ cpx mul_w16_9(cpx a) {
  return {-fmaf(a.x, kC1, a.y * kS1), -fmaf(a.y, kC1, -a.x * kS1)};
}

__device__ __forceinline__ void dft2(cpx &a, cpx &b) {
  cpx t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

// In-place 4-point DFT of (a0, a1, a2, a3), natural output order.
__device__ __forceinline__ void dft4(cpx &a0, cpx &a1, cpx &a2, cpx &a3) {
  cpx t0 = cadd(a0, a2), t1 = csub(a0, a2);
  cpx t2 = cadd(a1, a3), t3 = csub(a1, a3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, mul_mi(t3));
  a3 = cadd(t1, mul_pi(t3));
}

// In-place 8-point DFT: v[n] -> V[k], natural order.
// n = 2*n1 + n2; DFT4 over n1, twiddle W8^(n2*k1), DFT2 over n2.
__device__ __forceinline__ void dft8(cpx *v) {
  dft4(v[0], v[2], v[4], v[6]);  // n2 = 0 -> a0[k1] at v[0],v[2],v[4],v[6]
  dft4(v[1], v[3], v[5], v[7]);  // n2 = 1 -> a1[k1] at v[1],v[3],v[5],v[7]
  v[3] = mul_w8_1(v[3]);
  v[5] = mul_mi(v[5]);
  v[7] = mul_w8_3(v[7]);
  cpx o[8];
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    cpx a = v[2 * k1], b = v[2 * k1 + 1];
    o[k1] = cadd(a, b);
    o[k1 + 4] = csub(a, b);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = o[i];
}

// In-place 16-point DFT: v[n] -> V[k], natural order.
// n = 4*n1 + n2, k = k1 + 4*k2: DFT4 over n1, twiddle W16^(n2*k1), DFT4 over n2.
__device__ __forceinline__ void dft16(cpx *v) {
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
  // now v[n2 + 4*k1] = a[n2][k1]
  v[5] = mul_w16_1(v[5]);    // n2=1,k1=1 -> W^1
  v[9] = mul_w8_1(v[9]);     // n2=1,k1=2 -> W^2
  v[13] = mul_w16_3(v[13]);  // n2=1,k1=3 -> W^3
  v[6] = mul_w8_1(v[6]);     // n2=2,k1=1 -> W^2
  v[10] = mul_mi(v[10]);     // n2=2,k1=2 -> W^4
  v[14] = mul_w8_3(v[14]);   // n2=2,k1=3 -> W^6
  v[7] = mul_w16_3(v[7]);    // n2=3,k1=1 -> W^3
  v[11] = mul_w8_3(v[11]);   // n2=3,k1=2 -> W^6
  v[15] = mul_w16_9(v[15]);  // n2=3,k1=3 -> W^9
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // v[4*k1 + k2] = X[k1 + 4*k2]; transpose into natural order
  cpx o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) o[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = o[i];
}

template <int R>
__device__ __forceinline__ void dft(cpx *v) {
  if constexpr (R == 2) {
    dft2(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8(v);
  } else {
    static_assert(R == 16, "radix must be 2, 4, 8 or 16");
    dft16(v);
  }
}

}  // namespace mm
