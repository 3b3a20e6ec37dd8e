// Poseidon2 kernels: batch permutation, Merkle row hashing (PaddingFreeSponge
// rate 8, overwrite mode), 2-to-1 compression with mixed-height injection,
// FRI fold, and the device-side duplex challenger.
#include <cuda_runtime.h>

#include "field.cuh"
#include "internal.h"
#include "open.h"
#include "poseidon2.cuh"

namespace pico {

cudaError_t upload_p2_constants(int field, const uint32_t ext[8][16], const uint32_t* inte, int rounds_p,
                                const uint32_t diag[16]) {
  P2Constants h{};
  for (int r = 0; r < 8; r++)
    for (int j = 0; j < 16; j++) h.ext[r][j] = ext[r][j];
  for (int r = 0; r < rounds_p && r < 24; r++) h.inte[r] = inte[r];
  for (int j = 0; j < 16; j++) h.diag[j] = diag[j];
  return cudaMemcpyToSymbol(c_p2, &h, sizeof h, sizeof(P2Constants) * (field ? 1 : 0));
}

// ---------------------------------------------------------------------------
template <class F>
__global__ void k_permute(uint32_t* states, uint64_t n) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t s[16];
  uint4* p = reinterpret_cast<uint4*>(states + 16 * i);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint4 v = p[k];
    s[4 * k] = v.x;
    s[4 * k + 1] = v.y;
    s[4 * k + 2] = v.z;
    s[4 * k + 3] = v.w;
  }
  p2_permute<F>(s);
#pragma unroll
  for (int k = 0; k < 4; k++) p[k] = make_uint4(s[4 * k], s[4 * k + 1], s[4 * k + 2], s[4 * k + 3]);
}

// Absorb row r of the concatenated group into a zeroed sponge state
// (PaddingFreeSponge<_,16,8,8>: overwrite s[0..k) with each chunk of up to 8
// elements, permute after each chunk; hash.rs:40-52).
// Bounds guard of the row hashing: a read stays inside its row segment by
// construction (rows are bounded by the launch, columns by the segment
// widths), so the guard sits where the cursor moves to the next segment: a
// move past the last segment is skipped (reads as zero), recorded in
// g_hash_guard, and reported by the entry points after their final
// synchronisation.
__device__ GuardRecord g_hash_guard;
__device__ __forceinline__ void hash_guard_trip(unsigned long long seg, unsigned long long col) {
  if (atomicAdd(&g_hash_guard.count, 1ull) == 0) {
    g_hash_guard.tag = kGuardRowRead;
    g_hash_guard.offset = seg;
    g_hash_guard.extent = col;
    g_hash_guard.block = blockIdx.x;
    g_hash_guard.thread = threadIdx.x;
  }
}
template <class F>
__device__ __forceinline__ void hash_row_segs(const RowSeg* segs, uint32_t n_segs, uint32_t W, uint64_t r,
                                              uint32_t s[16]) {
  uint32_t seg = 0, col = 0;
  uint32_t segw = n_segs ? segs[0].width : 0u;
  const uint32_t* rowp = n_segs ? segs[0].ptr + r * segw : nullptr;
  for (uint32_t base = 0; base < W; base += 8) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (base + j < W) {
        while (col == segw && seg < n_segs) {
          seg++;
          col = 0;
          segw = seg < n_segs ? segs[seg].width : 0u;
          rowp = seg < n_segs ? segs[seg].ptr + r * segw : nullptr;
        }
        if (seg >= n_segs) {
          hash_guard_trip(seg, col);
          s[j] = 0;
        } else {
          s[j] = __ldg(rowp + col);
        }
        col++;
      }
    }
    p2_permute<F>(s);
  }
}

template <class F>
__device__ __forceinline__ void hash_row(const RowGroup& g, uint64_t r, uint32_t s[16], uint64_t rows) {
  (void)rows;
  hash_row_segs<F>(g.segs, g.n_segs, g.total_width, r, s);
}

__device__ __forceinline__ void store_digest(uint32_t* out, const uint32_t s[16]) {
  uint4* o = reinterpret_cast<uint4*>(out);
  o[0] = make_uint4(s[0], s[1], s[2], s[3]);
  o[1] = make_uint4(s[4], s[5], s[6], s[7]);
}

// Row digests of several height groups, one thread per row of any group:
// the groups' sponges, short and latency-bound when a group has few rows,
// run side by side instead of one launch after another.
template <class F>
__global__ void __launch_bounds__(256, 5) k_hash_groups(const __grid_constant__ GroupBatch b) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b.n_groups == 0 || b.n_groups > (uint32_t)kBatchGroups || t >= b.row_end[b.n_groups - 1]) return;
  uint32_t g = 0;
  while (g + 1 < b.n_groups && t >= b.row_end[g]) g++;
  const uint64_t r = t - (g ? b.row_end[g - 1] : 0ull);
  const uint32_t s0 = b.seg_begin[g], s1 = b.seg_begin[g + 1];
  if (s1 < s0 || s1 > (uint32_t)kBatchSegs) {
    hash_guard_trip(s0, s1);
    return;
  }
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = 0;
  hash_row_segs<F>(b.segs + s0, s1 - s0, b.width[g], r, s);
  store_digest(b.out[g] + 8 * r, s);
}

template <class F>
// (256, 5): 48 registers at 5/8 occupancy.  Measured on a 2^30-cell commit,
// leaf hashing takes 34.4 ms at (256, 8) (32 registers, full occupancy),
// 34.1 at (256, 6), 33.2 here and 33.4 at (256, 4): the permutation's
// instruction scheduling gains more from registers than from warps.
__global__ void __launch_bounds__(256, 5) k_hash_rows(const __grid_constant__ RowGroup g, uint64_t rows, uint32_t* out) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = 0;
  hash_row<F>(g, r, s, rows);
  store_digest(out + 8 * r, s);
}

// The same sponge, resumable: absorb the group's columns into a state that a
// previous call left in state_in (nullptr: the zero state), the first column
// going to rate position pos0 of the current chunk (the previous call's
// columns mod 8).  A call that is not the last stores the whole state to
// state_out, including a partly overwritten chunk that is not yet permuted;
// the last call permutes after its final (possibly partial) chunk, as the
// one-pass sponge does, and writes the digest.  Absorbing a row's matrices
// one call at a time gives the one-pass digest exactly.
template <class F>
__global__ void __launch_bounds__(256, 5)
    k_absorb_rows(const __grid_constant__ RowGroup g, uint64_t rows, uint32_t pos0, const uint32_t* state_in,
                  uint32_t* state_out, uint32_t* digest_out) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  uint32_t s[16];
  if (state_in) {
    // plain loads: state_in may be state_out (each thread rereads its own row)
    const uint4* p = reinterpret_cast<const uint4*>(state_in + 16 * r);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4 v = p[k];
      s[4 * k] = v.x;
      s[4 * k + 1] = v.y;
      s[4 * k + 2] = v.z;
      s[4 * k + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = 0;
  }
  const int W = (int)g.total_width;
  const int end = (int)pos0 + W;  // positions pos0 .. end-1 of the chunk sequence
  uint32_t seg = 0, col = 0;
  uint32_t segw = g.segs[0].width;
  const uint32_t* rowp = g.segs[0].ptr + r * segw;
  for (int base = 0; base < end; base += 8) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = base + j;  // chunk position; column c - pos0 of this call
      if (c >= (int)pos0 && c < end) {
        while (col == segw && seg < g.n_segs) {
          seg++;
          col = 0;
          segw = seg < g.n_segs ? g.segs[seg].width : 0u;
          rowp = g.segs[seg < g.n_segs ? seg : 0].ptr + r * segw;
        }
        if (seg >= g.n_segs) {
          hash_guard_trip(seg, col);
          s[j] = 0;
        } else {
          s[j] = __ldg(rowp + col);
        }
        col++;
      }
    }
    if (base + 8 <= end || digest_out) p2_permute<F>(s);
  }
  if (digest_out) {
    store_digest(digest_out + 8 * r, s);
  } else {
    uint4* o = reinterpret_cast<uint4*>(state_out + 16 * r);
#pragma unroll
    for (int k = 0; k < 4; k++) o[k] = make_uint4(s[4 * k], s[4 * k + 1], s[4 * k + 2], s[4 * k + 3]);
  }
}

// next[i] = compress(prev[2i], prev[2i+1]); where a matrix height meets this
// level, next[i] = compress(next[i], inj[i]) with inj[i] the digest of the
// concatenated rows i of those matrices (TruncatedPermutation, hash.rs:89-94;
// injection order of the verifier, fri.rs:389-436).
template <class F>
__global__ void __launch_bounds__(256)
    k_compress(const uint32_t* prev, uint32_t* next, uint64_t n, const uint32_t* inj) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t s[16];
  const uint4* p = reinterpret_cast<const uint4*>(prev + 16 * i);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint4 v = __ldg(p + k);
    s[4 * k] = v.x;
    s[4 * k + 1] = v.y;
    s[4 * k + 2] = v.z;
    s[4 * k + 3] = v.w;
  }
  p2_permute<F>(s);
  if (inj) {
    const uint4* q = reinterpret_cast<const uint4*>(inj + 8 * i);
    const uint4 a = __ldg(q), b = __ldg(q + 1);
    s[8] = a.x;
    s[9] = a.y;
    s[10] = a.z;
    s[11] = a.w;
    s[12] = b.x;
    s[13] = b.y;
    s[14] = b.z;
    s[15] = b.w;
    p2_permute<F>(s);
  }
  store_digest(next + 8 * i, s);
}

// ---------------------------------------------------------------------------
static inline unsigned blocks_for(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

// Four threads per state (the latency form).  Every thread of a launched warp
// takes part in the shuffles; threads past the last state permute zeros and
// store nothing.
template <class F>
__global__ void __launch_bounds__(256) k_permute_quad(uint32_t* states, uint64_t n) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t i = t >> 2;
  const uint32_t q = (uint32_t)(t & 3);
  const bool live = i < n;
  uint32_t v[4];
  if (live) {
    const uint4 a = reinterpret_cast<const uint4*>(states + 16 * i)[q];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  } else {
    v[0] = v[1] = v[2] = v[3] = 0;
  }
  p2_permute_quad<F>(v, q, 0xffffffffu);
  if (live) reinterpret_cast<uint4*>(states + 16 * i)[q] = make_uint4(v[0], v[1], v[2], v[3]);
}

cudaError_t launch_permute(int field, uint32_t* states, uint64_t n, cudaStream_t st, bool four_lanes) {
  if (n == 0) return cudaSuccess;
  if (four_lanes) {
    if (field == 0)
      k_permute_quad<KoalaBear><<<blocks_for(4 * n, 256), 256, 0, st>>>(states, n);
    else
      k_permute_quad<BabyBear><<<blocks_for(4 * n, 256), 256, 0, st>>>(states, n);
    return cudaGetLastError();
  }
  if (field == 0)
    k_permute<KoalaBear><<<blocks_for(n, 256), 256, 0, st>>>(states, n);
  else
    k_permute<BabyBear><<<blocks_for(n, 256), 256, 0, st>>>(states, n);
  return cudaGetLastError();
}

cudaError_t hash_guard_fetch(GuardRecord* dst, cudaStream_t st) {
  return cudaMemcpyFromSymbolAsync(dst, g_hash_guard, sizeof(GuardRecord), 0, cudaMemcpyDeviceToHost, st);
}
cudaError_t hash_guard_clear() {
  const GuardRecord z{};
  return cudaMemcpyToSymbol(g_hash_guard, &z, sizeof z);
}

// block: threads per CTA, 32 .. 256 (the kernels are bounded to 256).
cudaError_t launch_hash_rows(int field, const RowGroup& g, uint64_t rows, uint32_t* out, cudaStream_t st,
                             unsigned block) {
  if (rows == 0) return cudaSuccess;
  if (block < 32 || block > 256) block = 256;
  if (field == 0)
    k_hash_rows<KoalaBear><<<blocks_for(rows, block), block, 0, st>>>(g, rows, out);
  else
    k_hash_rows<BabyBear><<<blocks_for(rows, block), block, 0, st>>>(g, rows, out);
  return cudaGetLastError();
}

cudaError_t launch_hash_groups(int field, const GroupBatch& b, cudaStream_t st, unsigned block) {
  if (b.n_groups == 0) return cudaSuccess;
  if (b.n_groups > (uint32_t)kBatchGroups || b.n_segs > (uint32_t)kBatchSegs) return cudaErrorInvalidValue;
  const uint64_t rows = b.row_end[b.n_groups - 1];
  if (rows == 0) return cudaSuccess;
  if (block < 32 || block > 256) block = 256;
  if (field == 0)
    k_hash_groups<KoalaBear><<<blocks_for(rows, block), block, 0, st>>>(b);
  else
    k_hash_groups<BabyBear><<<blocks_for(rows, block), block, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_absorb_rows(int field, const RowGroup& g, uint64_t rows, uint32_t pos0, const uint32_t* state_in,
                               uint32_t* state_out, uint32_t* digest_out, cudaStream_t st, unsigned block) {
  if (rows == 0) return cudaSuccess;
  if (block < 32 || block > 256) block = 256;
  if (field == 0)
    k_absorb_rows<KoalaBear><<<blocks_for(rows, block), block, 0, st>>>(g, rows, pos0, state_in, state_out,
                                                                        digest_out);
  else
    k_absorb_rows<BabyBear><<<blocks_for(rows, block), block, 0, st>>>(g, rows, pos0, state_in, state_out,
                                                                       digest_out);
  return cudaGetLastError();
}

// The same compression, four threads per node (levels too small to fill the
// GPU, where one permutation's latency sets the launch's time).
template <class F>
__global__ void __launch_bounds__(256) k_compress_quad(const uint32_t* prev, uint32_t* next, uint64_t n,
                                                       const uint32_t* inj) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t i = t >> 2;
  const uint32_t q = (uint32_t)(t & 3);
  const bool live = i < n;
  uint32_t v[4] = {0, 0, 0, 0};
  if (live) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(prev + 16 * i) + q);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  p2_permute_quad<F>(v, q, 0xffffffffu);
  if (inj) {
    // compress(digest, injected digest): lanes 0, 1 keep the digest, lanes 2, 3 load the injection
    if (q >= 2) {
      if (live) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(inj + 8 * i) + (q - 2));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
      } else {
        v[0] = v[1] = v[2] = v[3] = 0;
      }
    }
    p2_permute_quad<F>(v, q, 0xffffffffu);
  }
  if (live && q < 2) reinterpret_cast<uint4*>(next + 8 * i)[q] = make_uint4(v[0], v[1], v[2], v[3]);
}

cudaError_t launch_compress(int field, const uint32_t* prev, uint32_t* next, uint64_t n_next,
                            const uint32_t* inj_digests, cudaStream_t st) {
  if (n_next == 0) return cudaSuccess;
  if (n_next <= kQuadMaxNodes) {
    if (field == 0)
      k_compress_quad<KoalaBear><<<blocks_for(4 * n_next, 256), 256, 0, st>>>(prev, next, n_next, inj_digests);
    else
      k_compress_quad<BabyBear><<<blocks_for(4 * n_next, 256), 256, 0, st>>>(prev, next, n_next, inj_digests);
    return cudaGetLastError();
  }
  if (field == 0)
    k_compress<KoalaBear><<<blocks_for(n_next, 256), 256, 0, st>>>(prev, next, n_next, inj_digests);
  else
    k_compress<BabyBear><<<blocks_for(n_next, 256), 256, 0, st>>>(prev, next, n_next, inj_digests);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FRI fold (TwoAdicFriGenericConfig::fold_matrix, mirrored by the verifier at
// vm/src/compiler/recursion/circuit/fri.rs:345-377): row r of the (len/2) x 2
// matrix (lo, hi) folds to
//   (lo + hi)/2 + (beta/2) * g_inv^rev(r) * (lo - hi),
// g = two_adic_generator(log len), rev over log(len/2) bits.  The pair is read
// at rows 2r, 2r+1 of cw; rg is its row in the whole codeword (r itself,
// except for one shard of a codeword split by rows).
template <class F>
__device__ __forceinline__ Ext4 fri_fold_row(const uint32_t* cw, uint32_t log_len, uint64_t r, const Ext4& hb,
                                             const TwiddleTables& tw, uint64_t rg) {
  using B = Fp<F>;
  using E = Ef<F>;
  // g_inv^rev(rg) = w_max^(-(rev(rg) << (S - log_len)))
  const uint32_t mask = (1u << F::TWO_ADICITY) - 1u;
  uint32_t e = (uint32_t)bitrev64(rg, (int)log_len - 1) << (F::TWO_ADICITY - log_len);
  e = (0u - e) & mask;
  uint32_t t = B::mul(__ldg(tw.hi + (e >> 14)), __ldg(tw.lo + (e & 0x3fffu)));
  const uint4 lo4 = __ldg(reinterpret_cast<const uint4*>(cw) + 2 * r);
  const uint4 hi4 = __ldg(reinterpret_cast<const uint4*>(cw) + 2 * r + 1);
  Ext4 lo{{lo4.x, lo4.y, lo4.z, lo4.w}}, hi{{hi4.x, hi4.y, hi4.z, hi4.w}};
  Ext4 sum = E::add(lo, hi), dif = E::sub(lo, hi);
  Ext4 res;
  Ext4 pd = E::mul(hb, E::scale(dif, t));
#pragma unroll
  for (int i = 0; i < 4; i++) res.c[i] = B::add(B::half(sum.c[i]), pd.c[i]);
  return res;
}

template <class F>
__device__ __forceinline__ Ext4 half_beta(const uint32_t* beta) {
  Ext4 hb;
#pragma unroll
  for (int i = 0; i < 4; i++) hb.c[i] = Fp<F>::half(__ldg(beta + i));
  return hb;
}

template <class F>
__global__ void k_fri_fold(const uint32_t* cw, uint32_t log_len, const uint32_t* beta, TwiddleTables tw,
                           uint32_t* out, const uint32_t* inject) {
  const uint64_t h = 1ull << (log_len - 1);
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= h) return;
  Ext4 res = fri_fold_row<F>(cw, log_len, r, half_beta<F>(beta), tw, r);
  if (inject) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(inject) + r);
    res = Ef<F>::add(res, Ext4{{v.x, v.y, v.z, v.w}});
  }
  reinterpret_cast<uint4*>(out)[r] = make_uint4(res.c[0], res.c[1], res.c[2], res.c[3]);
}

// Fold, then hash the next round's leaves in the same pass: thread k folds
// rows 2k and 2k+1 (adding the injected reduced opening), stores them, and
// hashes the pair as one 8-element leaf (one permutation: the rate block is
// the row, PaddingFreeSponge over 8 elements).
template <class F>
__global__ void __launch_bounds__(256) k_fri_fold_hash(const uint32_t* cw, uint32_t log_len, const uint32_t* beta,
                                                       TwiddleTables tw, uint32_t* out, const uint32_t* inject,
                                                       uint32_t* leaves) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= (1ull << (log_len - 2))) return;
  const Ext4 hb = half_beta<F>(beta);
  uint32_t s[16];
#pragma unroll
  for (int u = 0; u < 2; u++) {
    const uint64_t r = 2 * k + u;
    Ext4 res = fri_fold_row<F>(cw, log_len, r, hb, tw, r);
    if (inject) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(inject) + r);
      res = Ef<F>::add(res, Ext4{{v.x, v.y, v.z, v.w}});
    }
    reinterpret_cast<uint4*>(out)[r] = make_uint4(res.c[0], res.c[1], res.c[2], res.c[3]);
#pragma unroll
    for (int i = 0; i < 4; i++) s[4 * u + i] = res.c[i];
  }
#pragma unroll
  for (int i = 8; i < 16; i++) s[i] = 0;
  p2_permute<F>(s);
  uint4* lp = reinterpret_cast<uint4*>(leaves + 8 * k);
  lp[0] = make_uint4(s[0], s[1], s[2], s[3]);
  lp[1] = make_uint4(s[4], s[5], s[6], s[7]);
}

// One shard's part of k_fri_fold_hash for a codeword split by rows: the
// shard holds rows [2 row0, 2 row0 + 4 n_leaves) of the 2^log_len-row
// codeword at cw; it folds them into rows [row0, row0 + 2 n_leaves) (stored
// from out) and hashes their n_leaves leaves.
template <class F>
__global__ void __launch_bounds__(256) k_fri_fold_hash_rows(const uint32_t* cw, uint32_t log_len, uint64_t row0,
                                                            uint64_t n_leaves, const uint32_t* beta,
                                                            TwiddleTables tw, uint32_t* out, uint32_t* leaves) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n_leaves) return;
  const Ext4 hb = half_beta<F>(beta);
  uint32_t s[16];
#pragma unroll
  for (int u = 0; u < 2; u++) {
    const uint64_t r = 2 * k + u;
    const Ext4 res = fri_fold_row<F>(cw, log_len, r, hb, tw, row0 + r);
    reinterpret_cast<uint4*>(out)[r] = make_uint4(res.c[0], res.c[1], res.c[2], res.c[3]);
#pragma unroll
    for (int i = 0; i < 4; i++) s[4 * u + i] = res.c[i];
  }
#pragma unroll
  for (int i = 8; i < 16; i++) s[i] = 0;
  p2_permute<F>(s);
  uint4* lp = reinterpret_cast<uint4*>(leaves + 8 * k);
  lp[0] = make_uint4(s[0], s[1], s[2], s[3]);
  lp[1] = make_uint4(s[4], s[5], s[6], s[7]);
}

cudaError_t launch_fri_fold_hash_rows(int field, const uint32_t* cw, uint32_t log_len, uint64_t row0,
                                      uint64_t n_leaves, const uint32_t* beta, TwiddleTables tw, uint32_t* out,
                                      uint32_t* leaves, cudaStream_t st) {
  if (n_leaves == 0) return cudaSuccess;
  if (log_len < 2 || 2 * (row0 + 2 * n_leaves) > (1ull << log_len)) return cudaErrorInvalidValue;
  if (field == 0)
    k_fri_fold_hash_rows<KoalaBear><<<blocks_for(n_leaves, 256), 256, 0, st>>>(cw, log_len, row0, n_leaves, beta,
                                                                               tw, out, leaves);
  else
    k_fri_fold_hash_rows<BabyBear><<<blocks_for(n_leaves, 256), 256, 0, st>>>(cw, log_len, row0, n_leaves, beta,
                                                                              tw, out, leaves);
  return cudaGetLastError();
}

cudaError_t launch_fri_fold_hash(int field, const uint32_t* cw, uint32_t log_len, const uint32_t* beta,
                                 TwiddleTables tw, uint32_t* out, const uint32_t* inject, uint32_t* leaves,
                                 cudaStream_t st) {
  if (log_len < 2) return cudaErrorInvalidValue;
  const uint64_t n = 1ull << (log_len - 2);
  if (field == 0)
    k_fri_fold_hash<KoalaBear><<<blocks_for(n, 256), 256, 0, st>>>(cw, log_len, beta, tw, out, inject, leaves);
  else
    k_fri_fold_hash<BabyBear><<<blocks_for(n, 256), 256, 0, st>>>(cw, log_len, beta, tw, out, inject, leaves);
  return cudaGetLastError();
}

cudaError_t launch_fri_fold_tw(int field, const uint32_t* cw, uint32_t log_len, const uint32_t* beta,
                               TwiddleTables tw, uint32_t* out, cudaStream_t st, const uint32_t* inject) {
  uint64_t h = 1ull << (log_len - 1);
  if (field == 0)
    k_fri_fold<KoalaBear><<<blocks_for(h, 256), 256, 0, st>>>(cw, log_len, beta, tw, out, inject);
  else
    k_fri_fold<BabyBear><<<blocks_for(h, 256), 256, 0, st>>>(cw, log_len, beta, tw, out, inject);
  return cudaGetLastError();
}

// Duplex challenger (challenger.rs:89-115, 202-237), one thread.
template <class F>
__device__ void ch_duplex(DevChallenger* ch) {
  uint32_t s[16];
  for (int i = 0; i < 16; i++) s[i] = ch->sponge[i];
  for (uint32_t i = 0; i < ch->in_len; i++) s[i] = ch->in_buf[i];
  ch->in_len = 0;
  p2_permute<F>(s);
  for (int i = 0; i < 16; i++) ch->sponge[i] = s[i];
  for (int i = 0; i < 8; i++) ch->out_buf[i] = s[i];
  ch->out_len = 8;
}

template <class F>
__device__ void ch_observe(DevChallenger* ch, uint32_t v) {
  ch->out_len = 0;
  ch->in_buf[ch->in_len++] = v;
  if (ch->in_len == 8) ch_duplex<F>(ch);
}

template <class F>
__device__ uint32_t ch_sample(DevChallenger* ch) {
  if (ch->in_len != 0 || ch->out_len == 0) ch_duplex<F>(ch);
  return ch->out_buf[--ch->out_len];
}

template <class F>
__global__ void k_challenger_round(DevChallenger* ch, const uint32_t* root, uint32_t* beta_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < 8; i++) ch_observe<F>(ch, root[i]);
  for (int i = 0; i < 4; i++) beta_out[i] = ch_sample<F>(ch);
}

template <class F>
__global__ void k_challenger_observe(DevChallenger* ch, const uint32_t* vals, uint32_t n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (uint32_t i = 0; i < n; i++) ch_observe<F>(ch, vals[i]);
}

// The top of a Merkle tree in one block: `level` holds n_in <= 512 digests
// (a power of two); every level above it is computed in shared memory and
// written after it (the layer layout: each level follows the one below), up
// to the root.  With a challenger, thread 0 then observes the root and samples
// the EF4 challenge into beta_out (k_challenger_round's step).
constexpr uint32_t kTreeTopMax = 512;

template <class F>
__global__ void __launch_bounds__(256) k_tree_top(uint32_t* level, uint32_t n_in, DevChallenger* ch,
                                                  uint32_t* beta_out) {
  __shared__ uint32_t buf[kTreeTopMax * 8];
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < n_in * 8; i += blockDim.x) buf[i] = level[i];
  __syncthreads();
  uint32_t n = n_in;
  uint32_t* in = level;
  while (n > 1) {
    const uint32_t m = n >> 1;
    uint32_t* out = in + (size_t)n * 8;
    if (m > 64) {
      // one thread per node
      uint32_t st[16];
      if (tid < m) {
#pragma unroll
        for (int k = 0; k < 16; k++) st[k] = buf[16 * tid + k];
        p2_permute<F>(st);
      }
      __syncthreads();
      if (tid < m) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
          buf[8 * tid + k] = st[k];
          out[8 * tid + k] = st[k];
        }
      }
    } else {
      // four threads per node (4m <= 256): the latency form
      const uint32_t node = tid >> 2, q = tid & 3;
      uint32_t v[4];
      if (tid < 4 * m) {
        const unsigned mask = 4 * m >= 32 ? 0xffffffffu : ((1u << (4 * m)) - 1u);
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = buf[16 * node + 4 * q + k];
        p2_permute_quad<F>(v, q, mask);
      }
      __syncthreads();
      if (tid < 4 * m && q < 2) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          buf[8 * node + 4 * q + k] = v[k];
          out[8 * node + 4 * q + k] = v[k];
        }
      }
    }
    __syncthreads();
    in = out;
    n = m;
  }
  if (ch && tid == 0) {
    for (int i = 0; i < 8; i++) ch_observe<F>(ch, buf[i]);
    for (int i = 0; i < 4; i++) beta_out[i] = ch_sample<F>(ch);
  }
}

// Seven compression levels in one launch: CTA c reduces input nodes
// [128 c, 128 c + 128) of a level of n_in nodes to one node, four lanes per
// state, and writes every level it computes to the tree (level l + 1 follows
// level l, which holds n_in >> l nodes).  n_in is a multiple of 128.  Where
// inj.digests[l] is set, node i of computed level l is compressed once more
// with digest i of it (a commit's injected rows).  For the narrow levels of a
// tree this replaces seven latency-bound launches.
template <class F>
__global__ void __launch_bounds__(256) k_subtree_quad(uint32_t* level, uint32_t n_in,
                                                      const __grid_constant__ SubtreeInj inj) {
  __shared__ uint32_t buf[kSubtreeIn * 8];
  const uint32_t tid = threadIdx.x, c = blockIdx.x;
  if ((uint64_t)(c + 1) * kSubtreeIn > n_in) return;  // whole chunks only (the launcher checks n_in)
  const uint32_t* src = level + (size_t)c * kSubtreeIn * 8;
  for (uint32_t i = tid; i < kSubtreeIn * 8; i += blockDim.x) buf[i] = src[i];
  __syncthreads();
  uint32_t n = kSubtreeIn;  // this CTA's nodes at the current level
  uint32_t nl = n_in;       // the whole level's nodes
  uint32_t* in = level;
  uint32_t lvl = 0;         // levels computed so far
  while (n > 1) {
    const uint32_t m = n >> 1;
    uint32_t* out = in + (size_t)nl * 8;
    const uint32_t node = tid >> 2, q = tid & 3;
    const bool live = tid < 4 * m;
    uint32_t v[4];
    const uint32_t* d = inj.digests[lvl];
    if (live) {
      const unsigned mask = 4 * m >= 32 ? 0xffffffffu : ((1u << (4 * m)) - 1u);
#pragma unroll
      for (int k = 0; k < 4; k++) v[k] = buf[16 * node + 4 * q + k];
      p2_permute_quad<F>(v, q, mask);
      if (d) {
        // compress(node, injected digest): lanes 2, 3 load the injection
        if (q >= 2) {
          const uint4 a = __ldg(reinterpret_cast<const uint4*>(d + ((size_t)c * m + node) * 8) + (q - 2));
          v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        }
        p2_permute_quad<F>(v, q, mask);
      }
    }
    __syncthreads();
    if (live && q < 2) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        buf[8 * node + 4 * q + k] = v[k];
        out[((size_t)c * m + node) * 8 + 4 * q + k] = v[k];
      }
    }
    __syncthreads();
    in = out;
    nl >>= 1;
    n = m;
    lvl++;
  }
}

cudaError_t launch_subtree(int field, uint32_t* level, uint32_t n_in, const SubtreeInj& inj, cudaStream_t st) {
  if (n_in < kSubtreeIn || n_in % kSubtreeIn) return cudaErrorInvalidValue;
  if (field == 0)
    k_subtree_quad<KoalaBear><<<n_in / kSubtreeIn, 256, 0, st>>>(level, n_in, inj);
  else
    k_subtree_quad<BabyBear><<<n_in / kSubtreeIn, 256, 0, st>>>(level, n_in, inj);
  return cudaGetLastError();
}

cudaError_t launch_tree_top(int field, uint32_t* level, uint32_t n_in, DevChallenger* ch, uint32_t* beta_out,
                            cudaStream_t st) {
  if (n_in == 0 || n_in > kTreeTopMax || (n_in & (n_in - 1))) return cudaErrorInvalidValue;
  if (field == 0)
    k_tree_top<KoalaBear><<<1, 256, 0, st>>>(level, n_in, ch, beta_out);
  else
    k_tree_top<BabyBear><<<1, 256, 0, st>>>(level, n_in, ch, beta_out);
  return cudaGetLastError();
}

cudaError_t launch_challenger_round(int field, DevChallenger* ch, const uint32_t* root, uint32_t* beta_out,
                                    cudaStream_t st) {
  if (field == 0)
    k_challenger_round<KoalaBear><<<1, 32, 0, st>>>(ch, root, beta_out);
  else
    k_challenger_round<BabyBear><<<1, 32, 0, st>>>(ch, root, beta_out);
  return cudaGetLastError();
}

cudaError_t launch_challenger_observe(int field, DevChallenger* ch, const uint32_t* vals, uint32_t n,
                                      cudaStream_t st) {
  if (field == 0)
    k_challenger_observe<KoalaBear><<<1, 32, 0, st>>>(ch, vals, n);
  else
    k_challenger_observe<BabyBear><<<1, 32, 0, st>>>(ch, vals, n);
  return cudaGetLastError();
}

// Proof-of-work search (the challenger's grind; checked by check_witness,
// challenger.rs:210-221).  Observing candidate c and sampling always permutes
// once: the state with its pending inputs and c written over lanes
// 0..in_len, and the sample is lane 7 of the result (the last output popped).
// A candidate passes when the sample's canonical value has `bits` low zero
// bits; the smallest passing candidate of the launch wins (atomicMin).
template <class F>
__global__ void __launch_bounds__(256) k_grind(const DevChallenger* ch, uint32_t bits, uint32_t base,
                                               uint32_t count, uint32_t* best) {
  using B = Fp<F>;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (*reinterpret_cast<volatile uint32_t*>(best) != 0xffffffffu) return;  // found by an earlier launch
  if (k >= count) return;
  const uint64_t c = (uint64_t)base + k;
  if (c >= F::P) return;
  uint32_t s[16];
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = ch->sponge[i];
  const uint32_t n_in = ch->in_len;  // below 8: a full buffer is absorbed when it fills
  for (uint32_t i = 0; i < n_in && i < 8; i++) s[i] = ch->in_buf[i];
  const uint32_t v = B::to_monty((uint32_t)c);
#pragma unroll
  for (int i = 0; i < 8; i++)
    if ((uint32_t)i == n_in) s[i] = v;
  p2_permute<F>(s);
  const uint32_t mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
  if ((B::from_monty(s[7]) & mask) == 0) atomicMin(best, (uint32_t)c);
}

cudaError_t launch_grind(int field, const DevChallenger* ch, uint32_t bits, uint32_t base, uint32_t count,
                         uint32_t* best, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  const unsigned blocks = (count + 255) / 256;
  if (field == 0)
    k_grind<KoalaBear><<<blocks, 256, 0, st>>>(ch, bits, base, count, best);
  else
    k_grind<BabyBear><<<blocks, 256, 0, st>>>(ch, bits, base, count, best);
  return cudaGetLastError();
}

}  // namespace pico

namespace pico {

// Final polynomial of the commit phase when folding stops early: the
// remaining codeword holds 2^log_len evaluations in bit-reversed order; its
// coefficients over the subgroup are c_i = (1/len) sum_j v[rev(j)] w^(-ij).
// Coefficients at i >= 2^log_keep must vanish (low-degree check): a nonzero
// one sets *err.
template <class F>
__global__ void k_fri_final_poly(const uint32_t* cw, uint32_t log_len, uint32_t log_keep, TwiddleTables tw,
                                 uint32_t* coeffs, uint32_t* err) {
  using B = Fp<F>;
  const uint32_t len = 1u << log_len;
  const uint32_t mask = (1u << F::TWO_ADICITY) - 1u;
  const uint32_t len_inv = B::inv(B::to_monty(len));
  for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
    uint32_t acc[4] = {0, 0, 0, 0};
    for (uint32_t j = 0; j < len; j++) {
      uint32_t e = (uint32_t)(((uint64_t)i * j) & (len - 1)) << (F::TWO_ADICITY - log_len);
      e = (0u - e) & mask;
      const uint32_t wv = B::mul(__ldg(tw.hi + (e >> 14)), __ldg(tw.lo + (e & 0x3fffu)));
      const uint32_t* v = cw + 4 * bitrev32(j, log_len);
#pragma unroll
      for (int k = 0; k < 4; k++) acc[k] = B::add(acc[k], B::mul(v[k], wv));
    }
#pragma unroll
    for (int k = 0; k < 4; k++) acc[k] = B::mul(acc[k], len_inv);
    if (i < (1u << log_keep)) {
#pragma unroll
      for (int k = 0; k < 4; k++) coeffs[4 * i + k] = acc[k];
    } else if (acc[0] | acc[1] | acc[2] | acc[3]) {
      atomicExch(err, 1u);
    }
  }
}

cudaError_t launch_fri_final_poly(int field, const uint32_t* cw, uint32_t log_len, uint32_t log_keep,
                                  TwiddleTables tw, uint32_t* coeffs, uint32_t* err, cudaStream_t st) {
  if (field == 0)
    k_fri_final_poly<KoalaBear><<<1, 256, 0, st>>>(cw, log_len, log_keep, tw, coeffs, err);
  else
    k_fri_final_poly<BabyBear><<<1, 256, 0, st>>>(cw, log_len, log_keep, tw, coeffs, err);
  return cudaGetLastError();
}

}  // namespace pico
