// Monty-31 prime fields (KoalaBear, BabyBear) and their degree-4 binomial
// extensions, for host and device.
//
// Storage is Plonky3's MontyField31 form: an element x is held as the u32
// x * 2^32 mod p (the reference binds these types in
// vm/src/configs/stark_config/kb_poseidon2.rs:15 and bb_poseidon2.rs:15).
// Device values are kept canonical (< p) between operations.
//
//   KoalaBear p = 2^31 - 2^24 + 1, two-adicity 24, GENERATOR 3, EF4 x^4 = 3
//   BabyBear  p = 2^31 - 2^27 + 1, two-adicity 27, GENERATOR 31, EF4 x^4 = 11
// (generators: vm/src/compiler/recursion/ir/utils.rs:13-19; W:
// vm/src/primitives/consts.rs:107,134; S-box degrees and round counts:
// consts.rs:184-203).
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define PICO_HD __host__ __device__ __forceinline__
#else
#define PICO_HD inline
#endif

namespace pico {

constexpr uint32_t neg_inv_mod_2_32(uint32_t p) {
  // Newton iteration for p^-1 mod 2^32, then negate.
  uint32_t x = p;  // correct to 3 bits for odd p
  for (int i = 0; i < 5; i++) x *= 2u - p * x;
  return 0u - x;
}

struct KoalaBear {
  static constexpr int ID = 0;
  static constexpr uint32_t P = 0x7f000001u;
  static constexpr uint32_t NEG_PINV = neg_inv_mod_2_32(P);
  static constexpr uint32_t ONE = (uint32_t)((1ull << 32) % P);  // Monty(1)
  static constexpr uint32_t R2 = (uint32_t)(((unsigned __int128)1 << 64) % P);
  static constexpr int TWO_ADICITY = 24;
  static constexpr uint32_t GENERATOR = 3;
  static constexpr uint32_t W = 3;
  static constexpr int SBOX = 3;
  static constexpr int ROUNDS_P = 20;
  // p = C * 2^S + 1 (used by the shift-based multiply by 2^-k)
  static constexpr uint32_t PC = 127;
  static constexpr int PS = 24;
};

struct BabyBear {
  static constexpr int ID = 1;
  static constexpr uint32_t P = 0x78000001u;
  static constexpr uint32_t NEG_PINV = neg_inv_mod_2_32(P);
  static constexpr uint32_t ONE = (uint32_t)((1ull << 32) % P);
  static constexpr uint32_t R2 = (uint32_t)(((unsigned __int128)1 << 64) % P);
  static constexpr int TWO_ADICITY = 27;
  static constexpr uint32_t GENERATOR = 31;
  static constexpr uint32_t W = 11;
  static constexpr int SBOX = 7;
  static constexpr int ROUNDS_P = 13;
  static constexpr uint32_t PC = 15;
  static constexpr int PS = 27;
};

static_assert(KoalaBear::NEG_PINV == 0x7effffffu, "KB -p^-1");
static_assert(BabyBear::NEG_PINV == 0x77ffffffu, "BB -p^-1");

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return min(a, b); }
#endif

template <class F>
struct Fp {
  // a + b mod p for canonical inputs.
  static PICO_HD uint32_t add(uint32_t a, uint32_t b) {
    uint32_t r = a + b;
    uint32_t s = r - F::P;
    return s < r ? s : r;  // unsigned min: picks r - p when r >= p
  }
  static PICO_HD uint32_t sub(uint32_t a, uint32_t b) {
    uint32_t r = a - b;
    uint32_t s = r + F::P;
    return s < r ? s : r;  // when a < b, r wrapped high and r + p is the answer
  }
  static PICO_HD uint32_t neg(uint32_t a) { return sub(0u, a); }
  static PICO_HD uint32_t dbl(uint32_t a) { return add(a, a); }
  // Reduce r in [0, 2p) to [0, p).
  static PICO_HD uint32_t canon(uint32_t r) {
    uint32_t s = r - F::P;
    return s < r ? s : r;
  }
  // Montgomery reduction of t < 2^32 * p: returns t * 2^-32 mod p in [0, 2p).
  static PICO_HD uint32_t redc(uint64_t t) {
    uint32_t q = (uint32_t)t * F::NEG_PINV;
    uint64_t u = t + (uint64_t)q * F::P;
    return (uint32_t)(u >> 32);
  }
  // Montgomery product of canonical values: Monty(a) * Monty(b) -> Monty(ab).
  static PICO_HD uint32_t mul(uint32_t a, uint32_t b) { return canon(redc((uint64_t)a * b)); }
  static PICO_HD uint32_t sqr(uint32_t a) { return mul(a, a); }
  static PICO_HD uint32_t to_monty(uint32_t x) { return mul(x % F::P, F::R2); }
  static PICO_HD uint32_t from_monty(uint32_t x) { return canon(redc((uint64_t)x)); }
  static PICO_HD uint32_t pow(uint32_t a, uint64_t e) {
    uint32_t r = F::ONE;
    while (e) {
      if (e & 1) r = mul(r, a);
      a = mul(a, a);
      e >>= 1;
    }
    return r;
  }
  static PICO_HD uint32_t inv(uint32_t a) { return pow(a, (uint64_t)F::P - 2); }
  // a / 2 for canonical a.
  static PICO_HD uint32_t half(uint32_t a) { return (a + ((a & 1u) ? F::P : 0u)) >> 1; }
};

// Degree-4 binomial extension element, coefficients c0..c3 in Monty form.
struct Ext4 {
  uint32_t c[4];
};

template <class F>
struct Ef {
  using B = Fp<F>;
  static PICO_HD Ext4 add(const Ext4& a, const Ext4& b) {
    Ext4 r;
    for (int i = 0; i < 4; i++) r.c[i] = B::add(a.c[i], b.c[i]);
    return r;
  }
  static PICO_HD Ext4 sub(const Ext4& a, const Ext4& b) {
    Ext4 r;
    for (int i = 0; i < 4; i++) r.c[i] = B::sub(a.c[i], b.c[i]);
    return r;
  }
  static PICO_HD Ext4 scale(const Ext4& a, uint32_t s) {
    Ext4 r;
    for (int i = 0; i < 4; i++) r.c[i] = B::mul(a.c[i], s);
    return r;
  }
  // (a0 + a1 X + a2 X^2 + a3 X^3)(b0 + ...) mod X^4 - W: schoolbook, every
  // product reduced (Montgomery) and summed with modular additions.
  static PICO_HD Ext4 mul(const Ext4& a, const Ext4& b) {
    constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);  // Monty(W)
    // high part: X^4.. terms multiplied by W
    uint32_t h0 = B::mul(a.c[1], b.c[3]);
    h0 = B::add(h0, B::mul(a.c[2], b.c[2]));
    h0 = B::add(h0, B::mul(a.c[3], b.c[1]));
    uint32_t h1 = B::add(B::mul(a.c[2], b.c[3]), B::mul(a.c[3], b.c[2]));
    uint32_t h2 = B::mul(a.c[3], b.c[3]);
    Ext4 r;
    r.c[0] = B::add(B::mul(a.c[0], b.c[0]), B::mul(h0, Wm));
    r.c[1] = B::add(B::add(B::mul(a.c[0], b.c[1]), B::mul(a.c[1], b.c[0])), B::mul(h1, Wm));
    r.c[2] = B::add(B::add(B::mul(a.c[0], b.c[2]), B::mul(a.c[1], b.c[1])),
                    B::add(B::mul(a.c[2], b.c[0]), B::mul(h2, Wm)));
    r.c[3] = B::add(B::add(B::mul(a.c[0], b.c[3]), B::mul(a.c[1], b.c[2])),
                    B::add(B::mul(a.c[2], b.c[1]), B::mul(a.c[3], b.c[0])));
    return r;
  }
};

// Bit reversal of the low `bits` bits.
PICO_HD uint64_t bitrev64(uint64_t x, int bits) {
#if defined(__CUDA_ARCH__)
  return bits == 0 ? 0 : (__brevll(x) >> (64 - bits));
#else
  uint64_t r = 0;
  for (int i = 0; i < bits; i++) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
#endif
}
PICO_HD uint32_t bitrev32(uint32_t x, int bits) {
#if defined(__CUDA_ARCH__)
  return bits == 0 ? 0 : (__brev(x) >> (32 - bits));
#else
  return (uint32_t)bitrev64(x, bits);
#endif
}

}  // namespace pico
