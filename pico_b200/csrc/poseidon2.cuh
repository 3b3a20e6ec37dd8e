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

struct __align__(16) P2Constants {
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

// x^3 (KoalaBear) or x^7 (BabyBear) of a canonical x, canonical result.
// Montgomery products of canonical factors land below 1.5p, so a raw product
// can feed one more multiply before the single final reduction.
template <class F>
__device__ __forceinline__ uint32_t p2_sbox(uint32_t x) {
  using B = Fp<F>;
  if constexpr (F::SBOX == 3) {
    const uint32_t x2 = B::redc((uint64_t)x * x);  // < 1.5p
    return B::canon(B::redc((uint64_t)x2 * x));    // x2 * x < 1.5p^2 -> < 1.75p
  } else {
    const uint32_t x2 = B::canon(B::redc((uint64_t)x * x));
    const uint32_t x3 = B::canon(B::redc((uint64_t)x2 * x));
    const uint32_t x4 = B::redc((uint64_t)x2 * x2);  // < 1.5p
    return B::canon(B::redc((uint64_t)x4 * x3));     // < 1.75p
  }
}

// Reduce a 64-bit sum of at most 16 canonical values (< 2^35) to [0, p).
// With 2^31 = c (mod p): v = hi * 2^31 + lo == lo + hi * c.
template <class F>
__device__ __forceinline__ uint32_t p2_reduce_sum(uint64_t v) {
  using B = Fp<F>;
  constexpr uint32_t C = (uint32_t)((1ull << 31) % F::P);  // KB 2^24 - 1, BB 2^27 - 1
  const uint32_t hi = (uint32_t)(v >> 31), lo = (uint32_t)v & 0x7fffffffu;
  const uint32_t r = lo + hi * C;  // KB: < 2^31 + 2^28 < 2p; BB: < 2^31 + 15 (2^27 - 1) < 2^32
  if constexpr (F::ID == 0) {
    return B::canon(r);
  } else {
    return B::canon(r >= 2 * F::P ? r - F::P : r);
  }
}

// sum + D * x for D = +-2^-k and canonical x, without a Montgomery product.
// With p = c * 2^S + 1, 2^-k = -c * 2^(S-k), so for x = hi * 2^k + lo:
// x * 2^-k = hi - lo * c * 2^(S-k), and lo * c * 2^(S-k) < c * 2^S = p - 1.
template <class F, int KSH, bool NEG>
__device__ __forceinline__ uint32_t p2_add_pow2inv(uint32_t sum, uint32_t x) {
  using B = Fp<F>;
  constexpr uint32_t K = F::PC << (F::PS - KSH);
  const uint32_t hi = x >> KSH;
  const uint32_t m = (x & ((1u << KSH) - 1u)) * K;
  // +: hi + p - m in [1, p + 2^(31-k));  -: m - hi + p in (p - 2^(31-k), 2p)
  const uint32_t t = NEG ? (m - hi + F::P) : (hi + (F::P - m));
  return B::add(sum, B::canon(t));
}

// Internal layer s_i = s_i * D_i + sum(s).  The sum is a tree: pairs of
// canonical values fit 32 bits, the upper levels accumulate in 64 bits, one
// reduction at the end.
template <class F>
__device__ __forceinline__ void p2_internal_v2(uint32_t s[16], const uint32_t* diag) {
  using B = Fp<F>;
  uint32_t pr[8];
#pragma unroll
  for (int i = 0; i < 8; i++) pr[i] = s[2 * i] + s[2 * i + 1];
  const uint64_t q0 = (uint64_t)pr[0] + pr[1], q1 = (uint64_t)pr[2] + pr[3];
  const uint64_t q2 = (uint64_t)pr[4] + pr[5], q3 = (uint64_t)pr[6] + pr[7];
  const uint32_t sum = p2_reduce_sum<F>((q0 + q1) + (q2 + q3));
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
  // D[9..15]: KoalaBear 2^-8, 2^-3, 2^-24, -2^-8, -2^-3, -2^-4, -2^-24;
  //           BabyBear  2^-8, 2^-2, 2^-3, 2^-27, -2^-8, -2^-4, -2^-27.
  (void)diag;
  if constexpr (F::ID == 0) {
    s[9] = p2_add_pow2inv<F, 8, false>(sum, s[9]);
    s[10] = p2_add_pow2inv<F, 3, false>(sum, s[10]);
    s[11] = p2_add_pow2inv<F, 24, false>(sum, s[11]);
    s[12] = p2_add_pow2inv<F, 8, true>(sum, s[12]);
    s[13] = p2_add_pow2inv<F, 3, true>(sum, s[13]);
    s[14] = p2_add_pow2inv<F, 4, true>(sum, s[14]);
    s[15] = p2_add_pow2inv<F, 24, true>(sum, s[15]);
  } else {
    s[9] = p2_add_pow2inv<F, 8, false>(sum, s[9]);
    s[10] = p2_add_pow2inv<F, 2, false>(sum, s[10]);
    s[11] = p2_add_pow2inv<F, 3, false>(sum, s[11]);
    s[12] = p2_add_pow2inv<F, 27, false>(sum, s[12]);
    s[13] = p2_add_pow2inv<F, 8, true>(sum, s[13]);
    s[14] = p2_add_pow2inv<F, 4, true>(sum, s[14]);
    s[15] = p2_add_pow2inv<F, 27, true>(sum, s[15]);
  }
}

template <class F>
__device__ __forceinline__ void p2_full_round(uint32_t s[16], const uint32_t* rc) {
  using B = Fp<F>;
  uint32_t c[16];
#pragma unroll
  for (int j = 0; j < 16; j += 4) {
    const uint4 v = *reinterpret_cast<const uint4*>(rc + j);
    c[j] = v.x;
    c[j + 1] = v.y;
    c[j + 2] = v.z;
    c[j + 3] = v.w;
  }
#pragma unroll
  for (int j = 0; j < 16; j++) s[j] = p2_sbox<F>(B::add(s[j], c[j]));
  p2_external<F>(s);
}

// Rounds run as loops (not unrolled) so the permutation's code stays small
// enough for the instruction caches; each round reads its constants once.
template <class F>
__device__ __forceinline__ void p2_permute(uint32_t s[16]) {
  using B = Fp<F>;
  const P2Constants& C = c_p2[F::ID];
  p2_external<F>(s);
#pragma unroll 1
  for (int r = 0; r < 4; r++) p2_full_round<F>(s, C.ext[r]);
  uint32_t diag[16];
#pragma unroll
  for (int i = 9; i < 16; i++) diag[i] = C.diag[i];
#pragma unroll 1
  for (int r = 0; r < F::ROUNDS_P; r++) {
    s[0] = p2_sbox<F>(B::add(s[0], C.inte[r]));
    p2_internal_v2<F>(s, diag);
  }
#pragma unroll 1
  for (int r = 4; r < 8; r++) p2_full_round<F>(s, C.ext[r]);
}

// Four lanes per state (latency form).  Lane q of an aligned group of four
// holds s[4q .. 4q+3] in v[0..3]; all four lanes must call it together (the
// group exchanges values by shuffles within `mask`).  The 4x4 external block
// is local to a lane; its column sums and the internal layer's total cross
// the group by two xor-shuffles.  About 2.5x shorter than one thread running
// the whole permutation, at ~15% more instructions: for levels of a tree too
// small to fill the GPU, where a chain of dependent permutations sets the time.
template <class F>
__device__ __forceinline__ void p2_external_quad(uint32_t v[4], unsigned mask) {
  using B = Fp<F>;
  p2_m4<F>(v[0], v[1], v[2], v[3]);
  uint32_t t[4];
#pragma unroll
  for (int k = 0; k < 4; k++) t[k] = B::add(v[k], __shfl_xor_sync(mask, v[k], 1, 4));
#pragma unroll
  for (int k = 0; k < 4; k++) t[k] = B::add(t[k], __shfl_xor_sync(mask, t[k], 2, 4));
#pragma unroll
  for (int k = 0; k < 4; k++) v[k] = B::add(v[k], t[k]);
}

template <class F>
__device__ __forceinline__ void p2_permute_quad(uint32_t v[4], uint32_t q, unsigned mask) {
  using B = Fp<F>;
  const P2Constants& C = c_p2[F::ID];
  p2_external_quad<F>(v, mask);
#pragma unroll 1
  for (int r = 0; r < 4; r++) {
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = p2_sbox<F>(B::add(v[k], C.ext[r][4 * q + k]));
    p2_external_quad<F>(v, mask);
  }
  uint32_t d[4];
#pragma unroll
  for (int k = 0; k < 4; k++) d[k] = C.diag[4 * q + k];
#pragma unroll 1
  for (int r = 0; r < F::ROUNDS_P; r++) {
    if (q == 0) v[0] = p2_sbox<F>(B::add(v[0], C.inte[r]));
    // total of the 16 lanes: four local values (< 2^33 in 64 bits), then the group
    uint32_t t = p2_reduce_sum<F>((uint64_t)v[0] + v[1] + (uint64_t)v[2] + v[3]);
    t = B::add(t, __shfl_xor_sync(mask, t, 1, 4));
    t = B::add(t, __shfl_xor_sync(mask, t, 2, 4));
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = B::add(B::mul(v[k], d[k]), t);
  }
#pragma unroll 1
  for (int r = 4; r < 8; r++) {
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = p2_sbox<F>(B::add(v[k], C.ext[r][4 * q + k]));
    p2_external_quad<F>(v, mask);
  }
}

}  // namespace pico
