// Poseidon2 width-16 round layers shared by the device permutation
// (poseidon2.cuh) and the host challenger (api.cu): the external 4x4-block
// layer, the S-box and the internal layer.  Host and device therefore run the
// same arithmetic; only the round loop and where the constants live differ.
//
// External layer: 4x4 block M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] on
// each 4-lane block, then s_i += sum over blocks of lane i mod 4
// (gnark/poseidon2/poseidon2_koalabear.go:126-159).  Internal layer:
// s_i = s_i * D_i + sum(s) (poseidon2_koalabear.go:183-196) with D from
// vm/src/primitives/consts.rs:110-154.
#pragma once
#include "field.cuh"

namespace pico {

template <class F>
PICO_HD void p2_m4(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
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
PICO_HD void p2_external(uint32_t s[16]) {
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
PICO_HD uint32_t p2_sbox(uint32_t x) {
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
PICO_HD uint32_t p2_reduce_sum(uint64_t v) {
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
PICO_HD uint32_t p2_add_pow2inv(uint32_t sum, uint32_t x) {
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
PICO_HD void p2_internal_v2(uint32_t s[16], const uint32_t* diag) {
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

}  // namespace pico
