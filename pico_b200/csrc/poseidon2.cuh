// Poseidon2 width-16 permutation over KoalaBear / BabyBear, one state per
// thread, held in registers.
//
// Round structure (the reference's Poseidon2KoalaBear<16> / Poseidon2BabyBear<16>
// as initialised in vm/src/primitives/mod.rs:305-346 and restated in
// gnark/poseidon2/poseidon2_koalabear.go:71-98):
//   external linear layer; 4 full rounds; R_P partial rounds; 4 full rounds.
//   full round:    s_j += rc[r][j]; s_j = s_j^d; external layer
//   partial round: s_0 += rc_int[r]; s_0 = s_0^d; internal layer
// External layer: 4x4 block M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] on
// each 4-lane block, then s_i += sum over blocks of lane i mod 4
// (poseidon2_koalabear.go:126-159).  Internal layer: s_i = s_i * D_i + sum(s)
// (poseidon2_koalabear.go:183-196) with D from vm/src/primitives/consts.rs:110-154.
//
// Round constants live in __constant__ memory (uploaded at context creation
// in Montgomery form), so a different table can be installed at run time.
#pragma once
#include "field.cuh"

namespace pico {

struct P2Constants {
  uint32_t ext[8][16];  // full-round constants, Monty form: rounds 0..3 then the 4 final rounds
  uint32_t inte[24];    // partial-round constants (lane 0), Monty form
  uint32_t diag[16];    // internal diagonal D_i, Monty form
};

// Defined here: exactly one translation unit (p2_kernels.cu) includes this
// header; upload_p2_constants() there fills it for both fields.
__constant__ P2Constants c_p2[2];

template <class F>
__device__ __forceinline__ void p2_m4(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
  using B = Fp<F>;
  uint32_t t01 = B::add(a, b);
  uint32_t t23 = B::add(c, d);
  uint32_t t0123 = B::add(t01, t23);
  uint32_t t01123 = B::add(t0123, b);
  uint32_t t01233 = B::add(t0123, d);
  uint32_t nd = B::add(t01233, B::dbl(a));
  uint32_t nb = B::add(t01123, B::dbl(c));
  uint32_t na = B::add(t01123, t01);
  uint32_t nc = B::add(t01233, t23);
  a = na;
  b = nb;
  c = nc;
  d = nd;
}

template <class F>
__device__ __forceinline__ void p2_external(uint32_t s[16]) {
  using B = Fp<F>;
#pragma unroll
  for (int i = 0; i < 16; i += 4) p2_m4<F>(s[i], s[i + 1], s[i + 2], s[i + 3]);
  uint32_t sums[4];
#pragma unroll
  for (int k = 0; k < 4; k++) sums[k] = B::add(B::add(s[k], s[4 + k]), B::add(s[8 + k], s[12 + k]));
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = B::add(s[i], sums[i & 3]);
}

template <class F>
__device__ __forceinline__ uint32_t p2_sbox(uint32_t x) {
  using B = Fp<F>;
  if constexpr (F::SBOX == 3) {
    return B::mul(B::sqr(x), x);
  } else {
    uint32_t x2 = B::sqr(x);
    uint32_t x3 = B::mul(x2, x);
    uint32_t x4 = B::sqr(x2);
    return B::mul(x4, x3);
  }
}

template <class F>
__device__ __forceinline__ void p2_internal(uint32_t s[16]) {
  using B = Fp<F>;
  const P2Constants& C = c_p2[F::ID];
  uint32_t sum = B::add(s[0], s[1]);
#pragma unroll
  for (int i = 2; i < 16; i++) sum = B::add(sum, s[i]);
  // D[0..8] = -2, 1, 2, 1/2, 3, 4, -1/2, -3, -4 in both fields.
  s[0] = B::sub(sum, B::dbl(s[0]));
  s[1] = B::add(sum, s[1]);
  s[2] = B::add(sum, B::dbl(s[2]));
  s[3] = B::add(sum, B::half(s[3]));
  s[4] = B::add(sum, B::add(B::dbl(s[4]), s[4]));
  s[5] = B::add(sum, B::dbl(B::dbl(s[5])));
  s[6] = B::sub(sum, B::half(s[6]));
  s[7] = B::sub(sum, B::add(B::dbl(s[7]), s[7]));
  s[8] = B::sub(sum, B::dbl(B::dbl(s[8])));
#pragma unroll
  for (int i = 9; i < 16; i++) s[i] = B::add(sum, B::mul(s[i], C.diag[i]));
}

template <class F>
__device__ __forceinline__ void p2_permute(uint32_t s[16]) {
  using B = Fp<F>;
  const P2Constants& C = c_p2[F::ID];
  p2_external<F>(s);
#pragma unroll
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int j = 0; j < 16; j++) s[j] = p2_sbox<F>(B::add(s[j], C.ext[r][j]));
    p2_external<F>(s);
  }
#pragma unroll 4
  for (int r = 0; r < F::ROUNDS_P; r++) {
    s[0] = p2_sbox<F>(B::add(s[0], C.inte[r]));
    p2_internal<F>(s);
  }
#pragma unroll
  for (int r = 4; r < 8; r++) {
#pragma unroll
    for (int j = 0; j < 16; j++) s[j] = p2_sbox<F>(B::add(s[j], C.ext[r][j]));
    p2_external<F>(s);
  }
}

}  // namespace pico
