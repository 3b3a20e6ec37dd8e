// Poseidon2 width-16 permutation over KoalaBear / BabyBear, one state per
// thread, held in registers.
//
// Round structure (the reference's Poseidon2KoalaBear<16> / Poseidon2BabyBear<16>
// as initialised in vm/src/primitives/mod.rs:305-346 and restated in
// gnark/poseidon2/poseidon2_koalabear.go:71-98):
//   external linear layer; 4 full rounds; R_P partial rounds; 4 full rounds.
//   full round:    s_j += rc[r][j]; s_j = s_j^d; external layer
//   partial round: s_0 += rc_int[r]; s_0 = s_0^d; internal layer
// The layers themselves are in p2_layers.cuh (shared with the host).
//
// Round constants live in __constant__ memory (uploaded at context creation
// in Montgomery form), so a different table can be installed at run time.
#pragma once
#include "field.cuh"
#include "p2_layers.cuh"

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
