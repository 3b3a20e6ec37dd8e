// Kernels of the PCS opening (TwoAdicFriPcs::open, called at
// vm/src/machine/prover.rs:589; every step is fixed by the Pico verifier,
// vm/src/compiler/recursion/circuit/fri.rs:77-436):
//
//   k_inv_denoms     1 / (z - x_i) over the committed rows, x_i = g w_h^rev(i)
//   k_open_partial   opened values p(z) = (z^n - g^n)/(n g^(n-1)) *
//                    sum_k w_n^k / (z - g w_n^k) * y_k over each matrix's low
//                    coset (Plonky3's interpolate_coset): per-block partial sums
//   k_open_finalize  sums the partials and applies the scale
//   k_reduce         the reduced opening of one height:
//                    ro[i] = sum_z d_z[i] * (K_z - sum_(m,z) alpha^off(m,z) r_m[i]),
//                    r_m[i] = sum_j alpha^j M[i][j], K_z = sum alpha^off * r(p(z))
//   k_gather_queries the query records (rows and Merkle paths)
//
// Sums of products of field elements are accumulated lazily: a product of two
// canonical Montgomery values is below p^2 < 2^62; an accumulator folded with
// 2^32 = C (mod p), C = 2^32 mod p, stays below 2^32 (C + 1), and up to four
// more products fit in 64 bits before the next fold (checked below for both
// fields).  One Montgomery reduction per accumulated sum gives the Monty form
// of the sum of the underlying values.
#include <cuda_runtime.h>

#include "field.cuh"
#include "internal.h"
#include "open.h"

namespace pico {

template <class F>
struct Lazy {
  static constexpr uint64_t C = (1ull << 32) % F::P;
  static constexpr bool kFourFit =
      ((unsigned __int128)(C + 1) << 32) + 4 * (unsigned __int128)(F::P - 1) * (F::P - 1) <
      ((unsigned __int128)1 << 64);
  static_assert(kFourFit, "four products after a fold must fit 64 bits");
  static_assert(((C + 1) << 32) < ((uint64_t)F::P << 32), "a folded sum must be reducible by REDC");
  static __device__ __forceinline__ uint64_t fold(uint64_t x) { return (x >> 32) * C + (uint32_t)x; }
  static __device__ __forceinline__ uint32_t finish(uint64_t x) { return Fp<F>::canon(Fp<F>::redc(fold(x))); }
};

template <class F>
__device__ __forceinline__ uint32_t ompow(const TwiddleTables& tw, uint32_t E) {
  return Fp<F>::mul(__ldg(tw.hi + (E >> 14)), __ldg(tw.lo + (E & 0x3fffu)));
}

// Inverse through the quadratic subfield F[Y], Y = X^2 (Y^2 = W): with
// a = e + X o, a * (e - X o) = e^2 - Y o^2 =: b in F[Y], and b^-1 = conj(b) / N(b).
template <class F>
__device__ __forceinline__ Ext4 ef_inv(const Ext4& a) {
  using B = Fp<F>;
  constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);
  const uint32_t a0 = a.c[0], a1 = a.c[1], a2 = a.c[2], a3 = a.c[3];
  // e^2 = (a0^2 + W a2^2) + 2 a0 a2 Y ; o^2 = (a1^2 + W a3^2) + 2 a1 a3 Y
  const uint32_t e0 = B::add(B::mul(a0, a0), B::mul(Wm, B::mul(a2, a2)));
  const uint32_t e1 = B::dbl(B::mul(a0, a2));
  const uint32_t o0 = B::add(B::mul(a1, a1), B::mul(Wm, B::mul(a3, a3)));
  const uint32_t o1 = B::dbl(B::mul(a1, a3));
  // b = e^2 - Y o^2 = (e0 - W o1) + (e1 - o0) Y
  const uint32_t b0 = B::sub(e0, B::mul(Wm, o1));
  const uint32_t b1 = B::sub(e1, o0);
  const uint32_t nrm = B::sub(B::mul(b0, b0), B::mul(Wm, B::mul(b1, b1)));
  const uint32_t ni = B::inv(nrm);
  const uint32_t c = B::mul(b0, ni), d = B::neg(B::mul(b1, ni));  // b^-1 = c + d Y
  Ext4 r;
  r.c[0] = B::add(B::mul(a0, c), B::mul(Wm, B::mul(a2, d)));
  r.c[1] = B::neg(B::add(B::mul(a1, c), B::mul(Wm, B::mul(a3, d))));
  r.c[2] = B::add(B::mul(a0, d), B::mul(a2, c));
  r.c[3] = B::neg(B::add(B::mul(a1, d), B::mul(a3, c)));
  return r;
}

__device__ __forceinline__ Ext4 ld4(const uint4* p) {
  const uint4 v = __ldg(p);
  return Ext4{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ uint4 st4(const Ext4& a) { return make_uint4(a.c[0], a.c[1], a.c[2], a.c[3]); }

// ---------------------------------------------------------------------------
template <class F>
__global__ void k_inv_denoms(Ext4 z, uint32_t log_h, uint32_t g_monty, TwiddleTables tw, uint4* out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (1ull << log_h)) return;
  const uint32_t E = (uint32_t)bitrev64(i, (int)log_h) << (F::TWO_ADICITY - log_h);
  const uint32_t x = Fp<F>::mul(g_monty, ompow<F>(tw, E));
  Ext4 d = z;
  d.c[0] = Fp<F>::sub(d.c[0], x);
  out[i] = st4(ef_inv<F>(d));
}

cudaError_t launch_inv_denoms(int field, const uint32_t z[4], uint32_t log_h, TwiddleTables tw, uint32_t* out,
                              cudaStream_t st) {
  const uint64_t n = 1ull << log_h;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  Ext4 e{{z[0], z[1], z[2], z[3]}};
  if (field == 0)
    k_inv_denoms<KoalaBear><<<blocks, 256, 0, st>>>(e, log_h, Fp<KoalaBear>::to_monty(KoalaBear::GENERATOR), tw,
                                                     reinterpret_cast<uint4*>(out));
  else
    k_inv_denoms<BabyBear><<<blocks, 256, 0, st>>>(e, log_h, Fp<BabyBear>::to_monty(BabyBear::GENERATOR), tw,
                                                    reinterpret_cast<uint4*>(out));
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Opened values.  A block takes 2^log_rows consecutive rows of the low coset of
// one matrix (one descriptor: up to two points).  The per-row weights
// c_z[i] = w_n^rev(i) / (z - x_i) go to shared memory first; then each thread
// accumulates one column (narrow matrices: several rows per pass, summed in
// shared memory at the end; wide ones: column tiles of 256).
constexpr int kOpenThreads = 256;

template <class F, int NP>
__device__ void open_block(const OpenDesc& d, uint32_t chunk, const TwiddleTables& tw, const uint4* const* dinv,
                           uint4* partial, Ext4 (*coef)[2], uint32_t (*red)[2][4]) {
  const uint32_t R = 1u << d.log_rows;
  const uint64_t r0 = (uint64_t)chunk << d.log_rows;
  const uint32_t t = threadIdx.x;
  for (uint32_t r = t; r < R; r += kOpenThreads) {
    const uint64_t i = r0 + r;
    const uint32_t E = (uint32_t)bitrev64(i, (int)d.log_n) << (F::TWO_ADICITY - d.log_n);
    const uint32_t wk = ompow<F>(tw, E);
#pragma unroll
    for (int p = 0; p < NP; p++) coef[r][p] = Ef<F>::scale(ld4(dinv[p] + i), wk);
  }
  __syncthreads();
  const uint32_t w = d.w;
  const uint32_t* base = d.lde + r0 * w;
  if (w <= (uint32_t)kOpenThreads) {
    const uint32_t rpp = kOpenThreads / w;  // rows per pass
    const uint32_t ri = t / w, j = t - ri * w;
    uint64_t acc[NP][4] = {};
    if (ri < rpp) {
      uint32_t k = 0;
      for (uint32_t r = ri; r < R; r += rpp, k++) {
        const uint32_t y = __ldg(base + (uint64_t)r * w + j);
#pragma unroll
        for (int p = 0; p < NP; p++)
#pragma unroll
          for (int l = 0; l < 4; l++) acc[p][l] += (uint64_t)coef[r][p].c[l] * y;
        if ((k & 3) == 3) {
#pragma unroll
          for (int p = 0; p < NP; p++)
#pragma unroll
            for (int l = 0; l < 4; l++) acc[p][l] = Lazy<F>::fold(acc[p][l]);
        }
      }
    }
#pragma unroll
    for (int p = 0; p < NP; p++)
#pragma unroll
      for (int l = 0; l < 4; l++) red[t][p][l] = ri < rpp ? Lazy<F>::finish(acc[p][l]) : 0u;
    __syncthreads();
    if (t < w) {
#pragma unroll
      for (int p = 0; p < NP; p++) {
        Ext4 s{{0, 0, 0, 0}};
        for (uint32_t q = 0; q < rpp; q++) {
          const uint32_t* v = red[q * w + t][p];
          s = Ef<F>::add(s, Ext4{{v[0], v[1], v[2], v[3]}});
        }
        partial[d.part_off + ((uint64_t)chunk * NP + p) * w + t] = st4(s);
      }
    }
  } else {
    for (uint32_t j = t; j < w; j += kOpenThreads) {
      uint64_t acc[NP][4] = {};
      for (uint32_t r = 0; r < R; r++) {
        const uint32_t y = __ldg(base + (uint64_t)r * w + j);
#pragma unroll
        for (int p = 0; p < NP; p++)
#pragma unroll
          for (int l = 0; l < 4; l++) acc[p][l] += (uint64_t)coef[r][p].c[l] * y;
        if ((r & 3) == 3) {
#pragma unroll
          for (int p = 0; p < NP; p++)
#pragma unroll
            for (int l = 0; l < 4; l++) acc[p][l] = Lazy<F>::fold(acc[p][l]);
        }
      }
#pragma unroll
      for (int p = 0; p < NP; p++) {
        Ext4 s;
#pragma unroll
        for (int l = 0; l < 4; l++) s.c[l] = Lazy<F>::finish(acc[p][l]);
        partial[d.part_off + ((uint64_t)chunk * NP + p) * w + j] = st4(s);
      }
    }
  }
}

template <class F>
__global__ void __launch_bounds__(kOpenThreads) k_open_partial(const OpenDesc* descs, uint32_t n_desc,
                                                               const uint4* const* dinv_tables, TwiddleTables tw,
                                                               uint4* partial) {
  __shared__ Ext4 coef[kOpenMaxRows][2];
  __shared__ uint32_t red[kOpenThreads][2][4];
  // descriptor owning this block: the last with block0 <= blockIdx.x
  uint32_t lo = 0, hi = n_desc;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (descs[mid].block0 <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const OpenDesc d = descs[lo];
  const uint32_t chunk = blockIdx.x - d.block0;
  if (chunk >= (1u << (d.log_n - d.log_rows))) return;
  const uint4* dinv[2] = {dinv_tables[d.pt[0]], dinv_tables[d.pt[d.n_pts > 1 ? 1 : 0]]};
  if (d.n_pts == 2)
    open_block<F, 2>(d, chunk, tw, dinv, partial, coef, red);
  else
    open_block<F, 1>(d, chunk, tw, dinv, partial, coef, red);
}

template <class F>
__global__ void k_open_finalize(const OpenDesc* descs, const uint4* partial, const Ext4* scale, uint4* values) {
  const OpenDesc d = descs[blockIdx.x];
  const uint32_t chunks = 1u << (d.log_n - d.log_rows);
  for (uint32_t item = threadIdx.x; item < d.n_pts * d.w; item += blockDim.x) {
    const uint32_t p = item / d.w, j = item - p * d.w;
    Ext4 s{{0, 0, 0, 0}};
    for (uint32_t c = 0; c < chunks; c++) s = Ef<F>::add(s, ld4(partial + d.part_off + ((uint64_t)c * d.n_pts + p) * d.w + j));
    values[d.out_off[p] + j] = st4(Ef<F>::mul(s, scale[2 * blockIdx.x + p]));
  }
}

cudaError_t launch_open_values(int field, const OpenDesc* descs, uint32_t n_desc, uint32_t n_blocks,
                               const uint32_t* const* dinv_tables, TwiddleTables tw, uint32_t* partial,
                               const uint32_t* scale, uint32_t* values, cudaStream_t st) {
  if (n_desc == 0) return cudaSuccess;
  auto dt = reinterpret_cast<const uint4* const*>(dinv_tables);
  auto pa = reinterpret_cast<uint4*>(partial);
  auto sc = reinterpret_cast<const Ext4*>(scale);
  auto va = reinterpret_cast<uint4*>(values);
  if (field == 0) {
    k_open_partial<KoalaBear><<<n_blocks, kOpenThreads, 0, st>>>(descs, n_desc, dt, tw, pa);
    k_open_finalize<KoalaBear><<<n_desc, 256, 0, st>>>(descs, pa, sc, va);
  } else {
    k_open_partial<BabyBear><<<n_blocks, kOpenThreads, 0, st>>>(descs, n_desc, dt, tw, pa);
    k_open_finalize<BabyBear><<<n_desc, 256, 0, st>>>(descs, pa, sc, va);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Reduced opening of one height: one thread per row.
template <class F, int NS>
__global__ void __launch_bounds__(256) k_reduce(ReduceHeight h) {
  using E = Ef<F>;
  using L = Lazy<F>;
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (1ull << h.log_h)) return;
  uint64_t acc[NS][4] = {};
  for (uint32_t m = 0; m < h.n_mats; m++) {
    const ReduceMat M = h.mats[m];
    const uint32_t* row = M.lde + i * M.w;
    const uint4* coef = h.apow + (M.multi ? 0u : M.off);
    uint64_t t[4] = {0, 0, 0, 0};
    uint32_t j = 0;
    for (; j + 4 <= M.w; j += 4) {
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t y = __ldg(row + j + u);
        const uint4 c = __ldg(coef + j + u);
        t[0] += (uint64_t)c.x * y;
        t[1] += (uint64_t)c.y * y;
        t[2] += (uint64_t)c.z * y;
        t[3] += (uint64_t)c.w * y;
      }
#pragma unroll
      for (int l = 0; l < 4; l++) t[l] = L::fold(t[l]);
    }
    for (; j < M.w; j++) {
      const uint32_t y = __ldg(row + j);
      const uint4 c = __ldg(coef + j);
      t[0] += (uint64_t)c.x * y;
      t[1] += (uint64_t)c.y * y;
      t[2] += (uint64_t)c.z * y;
      t[3] += (uint64_t)c.w * y;
    }
    if (!M.multi) {
#pragma unroll
      for (int q = 0; q < NS; q++)
        if (q == (int)M.slot) {
#pragma unroll
          for (int l = 0; l < 4; l++) acc[q][l] = L::fold(L::fold(acc[q][l]) + L::fold(t[l]));
        }
      continue;
    }
    // r = sum_j alpha^j M[i][j]; each (slot, alpha^off) term adds alpha^off * r
    Ext4 r;
#pragma unroll
    for (int l = 0; l < 4; l++) r.c[l] = L::finish(t[l]);
    for (uint32_t k = 0; k < M.n_terms; k++) {
      const ReduceTerm T = h.terms[M.term0 + k];
      const Ext4 a = ld4(h.apow + T.off);
      constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);
      const uint32_t wa1 = Fp<F>::mul(a.c[1], Wm), wa2 = Fp<F>::mul(a.c[2], Wm), wa3 = Fp<F>::mul(a.c[3], Wm);
#pragma unroll
      for (int q = 0; q < NS; q++)
        if (q == (int)T.slot) {
          uint64_t* s = acc[q];
          s[0] = L::fold(s[0]);
          s[1] = L::fold(s[1]);
          s[2] = L::fold(s[2]);
          s[3] = L::fold(s[3]);
          s[0] += (uint64_t)a.c[0] * r.c[0] + (uint64_t)wa1 * r.c[3] + (uint64_t)wa2 * r.c[2] + (uint64_t)wa3 * r.c[1];
          s[1] += (uint64_t)a.c[0] * r.c[1] + (uint64_t)a.c[1] * r.c[0] + (uint64_t)wa2 * r.c[3] + (uint64_t)wa3 * r.c[2];
          s[2] += (uint64_t)a.c[0] * r.c[2] + (uint64_t)a.c[1] * r.c[1] + (uint64_t)a.c[2] * r.c[0] + (uint64_t)wa3 * r.c[3];
          s[3] += (uint64_t)a.c[0] * r.c[3] + (uint64_t)a.c[1] * r.c[2] + (uint64_t)a.c[2] * r.c[1] + (uint64_t)a.c[3] * r.c[0];
        }
    }
  }
  Ext4 res{{0, 0, 0, 0}};
  if (h.accumulate) res = ld4(h.ro + i);
#pragma unroll
  for (int q = 0; q < NS; q++) {
    Ext4 s;
#pragma unroll
    for (int l = 0; l < 4; l++) s.c[l] = L::finish(acc[q][l]);
    res = E::add(res, E::mul(ld4(h.dinv[q] + i), E::sub(h.K[q], s)));
  }
  h.ro[i] = st4(res);
}

template <class F>
static cudaError_t launch_reduce_t(const ReduceHeight& h, cudaStream_t st) {
  const uint64_t n = 1ull << h.log_h;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  switch (h.n_slots) {
    case 1: k_reduce<F, 1><<<blocks, 256, 0, st>>>(h); break;
    case 2: k_reduce<F, 2><<<blocks, 256, 0, st>>>(h); break;
    case 3: k_reduce<F, 3><<<blocks, 256, 0, st>>>(h); break;
    case 4: k_reduce<F, 4><<<blocks, 256, 0, st>>>(h); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_reduce(int field, const ReduceHeight& h, cudaStream_t st) {
  return field == 0 ? launch_reduce_t<KoalaBear>(h, st) : launch_reduce_t<BabyBear>(h, st);
}

// ---------------------------------------------------------------------------
// Query records: one block per query, one warp per segment.
__global__ void k_gather_queries(const QuerySeg* segs, uint32_t n_segs, const uint32_t* indices, uint64_t query_words,
                                 uint32_t* out) {
  const uint64_t idx = indices[blockIdx.x];
  uint32_t* rec = out + blockIdx.x * query_words;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (uint32_t s = warp; s < n_segs; s += nw) {
    const QuerySeg q = segs[s];
    const uint64_t k = idx >> q.shift;
    const uint32_t* src;
    uint32_t len;
    if (q.kind == kSegRow) {
      src = q.base + k * q.width;
      len = q.width;
    } else if (q.kind == kSegDigest) {
      src = q.base + (q.level_off + (k ^ 1ull)) * 8;
      len = 8;
    } else {
      src = q.base + (k ^ 1ull) * 4;
      len = 4;
    }
    for (uint32_t u = lane; u < len; u += 32) rec[q.dst + u] = src[u];
  }
}

cudaError_t launch_gather_queries(const QuerySeg* segs, uint32_t n_segs, const uint32_t* indices, uint32_t n_queries,
                                  uint64_t query_words, uint32_t* out, cudaStream_t st) {
  if (n_queries == 0) return cudaSuccess;
  k_gather_queries<<<n_queries, 256, 0, st>>>(segs, n_segs, indices, query_words, out);
  return cudaGetLastError();
}

}  // namespace pico
