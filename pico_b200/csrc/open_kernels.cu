// Kernels of the PCS opening (TwoAdicFriPcs::open, called at
// vm/src/machine/prover.rs:589; every step is fixed by the Pico verifier,
// vm/src/compiler/recursion/circuit/fri.rs:77-436):
//
//   k_inv_denoms     1 / (z - x_i) over the committed rows, x_i = g w_h^rev(i)
//   k_open_partial   opened values p(z) = (z^n - g^n)/(n g^(n-1)) *
//                    sum_k w_n^k / (z - g w_n^k) * y_k over each matrix's low
//                    coset (Plonky3's interpolate_coset): per-block partial sums
//   k_open_finalize  sums the partials and applies the scale
//   k_reduce         per point z of a height, over the low coset only (the
//                    first n committed rows): S_z[i] = sum_(m,z) alpha^off(m,z) r_m[i],
//                    r_m[i] = sum_j alpha^j M[i][j]
//   k_reduce_combine the reduced opening on the low coset,
//                    ro = sum_z (K_z - S_z) / (z - x), K_z = sum alpha^off * sum_j
//                    alpha^j p_j(z) = S_z(z): a polynomial of degree < n, so the
//                    ordinary LDE kernels extend it to the committed rows
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
  // acc += a * b (one 32x32 -> 64-bit multiply-add)
  static __device__ __forceinline__ void mac(uint64_t& acc, uint32_t a, uint32_t b) {
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc) : "r"(a), "r"(b));
  }
  // hi * C + lo: congruent mod p, below 2^32 (C + 1)
  static __device__ __forceinline__ uint64_t fold(uint64_t x) {
    uint32_t lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=r"(lo), "=r"(hi) : "l"(x));
    uint64_t r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(hi), "n"((uint32_t)C), "l"((uint64_t)lo));
    return r;
  }
  static __device__ __forceinline__ uint32_t finish(uint64_t x) { return Fp<F>::canon(Fp<F>::redc(fold(x))); }
};

template <class F>
__device__ __forceinline__ uint32_t ompow(const TwiddleTables& tw, uint32_t E) {
  return Fp<F>::mul(__ldg(tw.hi + (E >> 14)), __ldg(tw.lo + (E & 0x3fffu)));
}

__device__ __forceinline__ Ext4 ld4(const uint4* p) {
  const uint4 v = __ldg(p);
  return Ext4{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ uint4 st4(const Ext4& a) { return make_uint4(a.c[0], a.c[1], a.c[2], a.c[3]); }

// ---------------------------------------------------------------------------
// 1/(z - x_i) for eight consecutive rows per thread.  Each inverse goes through
// the quadratic subfield F[Y], Y = X^2 (Y^2 = W): with a = e + X o,
// a (e - X o) = e^2 - Y o^2 =: b in F[Y] and b^-1 = conj(b) / N(b), N(b) in F.
// The eight norms share one base-field inversion (Montgomery's simultaneous
// inversion: prefix products, one inverse, back-substitution).
constexpr uint32_t kInvPerThread = 8;

template <class F>
__global__ void __launch_bounds__(256) k_inv_denoms(Ext4 z, uint32_t log_h, uint32_t g_monty, TwiddleTables tw,
                                                    uint4* out) {
  using B = Fp<F>;
  constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);
  const uint64_t n = 1ull << log_h;
  const uint64_t i0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * kInvPerThread;
  if (i0 >= n) return;
  const uint32_t cnt = n - i0 < kInvPerThread ? (uint32_t)(n - i0) : kInvPerThread;
  uint32_t b0[kInvPerThread], b1[kInvPerThread], nrm[kInvPerThread], pre[kInvPerThread];
  Ext4 a[kInvPerThread];
  uint32_t run = F::ONE;
#pragma unroll
  for (uint32_t k = 0; k < kInvPerThread; k++) {
    const uint64_t i = i0 + (k < cnt ? k : 0);
    const uint32_t E = (uint32_t)bitrev64(i, (int)log_h) << (F::TWO_ADICITY - log_h);
    a[k] = z;
    a[k].c[0] = B::sub(z.c[0], B::mul(g_monty, ompow<F>(tw, E)));
    const uint32_t x0 = a[k].c[0], x1 = a[k].c[1], x2 = a[k].c[2], x3 = a[k].c[3];
    const uint32_t e0 = B::add(B::mul(x0, x0), B::mul(Wm, B::mul(x2, x2)));
    const uint32_t e1 = B::dbl(B::mul(x0, x2));
    const uint32_t o0 = B::add(B::mul(x1, x1), B::mul(Wm, B::mul(x3, x3)));
    const uint32_t o1 = B::dbl(B::mul(x1, x3));
    b0[k] = B::sub(e0, B::mul(Wm, o1));
    b1[k] = B::sub(e1, o0);
    nrm[k] = B::sub(B::mul(b0[k], b0[k]), B::mul(Wm, B::mul(b1[k], b1[k])));
    pre[k] = run;  // product of the norms before k
    run = B::mul(run, nrm[k]);
  }
  uint32_t inv = B::inv(run);
#pragma unroll
  for (int k = kInvPerThread - 1; k >= 0; k--) {
    const uint32_t ni = B::mul(inv, pre[k]);  // 1 / nrm[k]
    inv = B::mul(inv, nrm[k]);
    const uint32_t c = B::mul(b0[k], ni), d = B::neg(B::mul(b1[k], ni));
    const uint32_t x0 = a[k].c[0], x1 = a[k].c[1], x2 = a[k].c[2], x3 = a[k].c[3];
    Ext4 r;
    r.c[0] = B::add(B::mul(x0, c), B::mul(Wm, B::mul(x2, d)));
    r.c[1] = B::neg(B::add(B::mul(x1, c), B::mul(Wm, B::mul(x3, d))));
    r.c[2] = B::add(B::mul(x0, d), B::mul(x2, c));
    r.c[3] = B::neg(B::add(B::mul(x1, d), B::mul(x3, c)));
    if ((uint32_t)k < cnt) out[i0 + k] = st4(r);
  }
}

cudaError_t launch_inv_denoms(int field, const uint32_t z[4], uint32_t log_h, TwiddleTables tw, uint32_t* out,
                              cudaStream_t st) {
  const uint64_t n = 1ull << log_h;
  const uint64_t threads = (n + kInvPerThread - 1) / kInvPerThread;
  const unsigned blocks = (unsigned)((threads + 255) / 256);
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
  const uint32_t R = 1u << d.log_rows;  // rows of this block; above kOpenMaxRows only when w <= kOpenThreads
  const uint64_t r0 = (uint64_t)chunk << d.log_rows;
  const uint32_t t = threadIdx.x;
  const uint32_t w = d.w;
  const bool narrow = w <= (uint32_t)kOpenThreads;
  const uint32_t rpp = narrow ? kOpenThreads / w : 1;  // rows per pass (narrow form)
  const uint32_t ri = narrow ? t / w : 0, j = narrow ? t - ri * w : t;
  uint64_t acc[NP][4] = {};
  for (uint32_t sub = 0; sub < R; sub += kOpenMaxRows) {
    const uint32_t Rs = min(R - sub, kOpenMaxRows);
    for (uint32_t r = t; r < Rs; r += kOpenThreads) {
      const uint64_t i = r0 + sub + r;
      const uint32_t E = (uint32_t)bitrev64(i, (int)d.log_n) << (F::TWO_ADICITY - d.log_n);
      const uint32_t wk = ompow<F>(tw, E);
#pragma unroll
      for (int p = 0; p < NP; p++) coef[r][p] = Ef<F>::scale(ld4(dinv[p] + i), wk);
    }
    __syncthreads();
    const uint32_t* base = d.lde + (r0 + sub) * w;
    if (narrow) {
      if (ri < rpp) {
        // eight rows per batch, their loads issued together
        for (uint32_t r = ri; r < Rs; r += 8 * rpp) {
          uint32_t y[8];
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const uint32_t rr = r + u * rpp;
            y[u] = rr < Rs ? __ldg(base + (uint64_t)rr * w + j) : 0u;
          }
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const uint32_t rr = min(r + u * rpp, Rs - 1);  // past the end: y = 0 adds nothing
#pragma unroll
            for (int p = 0; p < NP; p++)
#pragma unroll
              for (int l = 0; l < 4; l++) Lazy<F>::mac(acc[p][l], coef[rr][p].c[l], y[u]);
            if ((u & 3) == 3) {
#pragma unroll
              for (int p = 0; p < NP; p++)
#pragma unroll
                for (int l = 0; l < 4; l++) acc[p][l] = Lazy<F>::fold(acc[p][l]);
            }
          }
        }
      }
    } else {
      // wide: one sub-chunk only (R <= kOpenMaxRows), column tiles of kOpenThreads
      for (uint32_t jj = t; jj < w; jj += kOpenThreads) {
        uint64_t a2[NP][4] = {};
        for (uint32_t r = 0; r < Rs; r += 8) {
          uint32_t y[8];
#pragma unroll
          for (int u = 0; u < 8; u++) y[u] = r + u < Rs ? __ldg(base + (uint64_t)(r + u) * w + jj) : 0u;
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const uint32_t rr = min(r + u, Rs - 1);
#pragma unroll
            for (int p = 0; p < NP; p++)
#pragma unroll
              for (int l = 0; l < 4; l++) Lazy<F>::mac(a2[p][l], coef[rr][p].c[l], y[u]);
            if ((u & 3) == 3) {
#pragma unroll
              for (int p = 0; p < NP; p++)
#pragma unroll
                for (int l = 0; l < 4; l++) a2[p][l] = Lazy<F>::fold(a2[p][l]);
            }
          }
        }
#pragma unroll
        for (int p = 0; p < NP; p++) {
          Ext4 s;
#pragma unroll
          for (int l = 0; l < 4; l++) s.c[l] = Lazy<F>::finish(a2[p][l]);
          partial[d.part_off + ((uint64_t)chunk * NP + p) * w + jj] = st4(s);
        }
      }
    }
    __syncthreads();
  }
  if (!narrow) return;
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
}

template <class F>
__global__ void __launch_bounds__(kOpenThreads, 3) k_open_partial(const OpenDesc* descs, uint32_t n_desc,
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

// One warp per output value: the lanes stride over the blocks' partial sums,
// then a shuffle tree adds the 32 lane sums.
template <class F>
__global__ void k_open_finalize(const OpenDesc* descs, const uint4* partial, const Ext4* scale, uint4* values) {
  const OpenDesc* d = descs + blockIdx.y;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t item = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t n_pts = d->n_pts, w = d->w;
  if (item >= n_pts * w) return;
  const uint32_t chunks = 1u << (d->log_n - d->log_rows);
  const uint32_t p = item / w, j = item - p * w;
  const uint4* src = partial + d->part_off + (uint64_t)p * w + j;
  const uint64_t stride = (uint64_t)n_pts * w;
  Ext4 s{{0, 0, 0, 0}};
  for (uint32_t c = lane; c < chunks; c += 32) s = Ef<F>::add(s, ld4(src + c * stride));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Ext4 t;
#pragma unroll
    for (int l = 0; l < 4; l++) t.c[l] = __shfl_xor_sync(0xffffffffu, s.c[l], o);
    s = Ef<F>::add(s, t);
  }
  if (lane == 0) values[d->out_off[p] + j] = st4(Ef<F>::mul(s, scale[2 * blockIdx.y + p]));
}

cudaError_t launch_open_values(int field, const OpenDesc* descs, uint32_t n_desc, uint32_t n_blocks,
                               uint32_t max_items, const uint32_t* const* dinv_tables, TwiddleTables tw,
                               uint32_t* partial, const uint32_t* scale, uint32_t* values, cudaStream_t st) {
  if (n_desc == 0) return cudaSuccess;
  const unsigned fin_tiles = (max_items + 7) / 8;  // eight warps (values) per block
  auto dt = reinterpret_cast<const uint4* const*>(dinv_tables);
  auto pa = reinterpret_cast<uint4*>(partial);
  auto sc = reinterpret_cast<const Ext4*>(scale);
  auto va = reinterpret_cast<uint4*>(values);
  if (field == 0) {
    k_open_partial<KoalaBear><<<n_blocks, kOpenThreads, 0, st>>>(descs, n_desc, dt, tw, pa);
    k_open_finalize<KoalaBear><<<dim3(fin_tiles, n_desc), 256, 0, st>>>(descs, pa, sc, va);
  } else {
    k_open_partial<BabyBear><<<n_blocks, kOpenThreads, 0, st>>>(descs, n_desc, dt, tw, pa);
    k_open_finalize<BabyBear><<<dim3(fin_tiles, n_desc), 256, 0, st>>>(descs, pa, sc, va);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Reduced opening of one height.  Lane l of a warp owns row row0 + l; the
// warp stages its 32 rows through shared memory in tiles of 32 columns, loaded
// with coalesced reads (a matrix of at most 32 columns as one contiguous block
// of 32 rows), and each lane reads its row back across the banks (row stride
// 33 words).  The alpha powers are read by all lanes at the same address.
constexpr int kReduceWarps = 4;
constexpr int kTileStride = 36;  // words per tile row: 16-byte aligned; eight lanes' 16-byte reads cover the 32 banks
constexpr int kTileWords = 32 * kTileStride;        // data part of a tile buffer
constexpr int kTileBufWords = kTileWords + 32 * 4;   // + the 32 alpha powers of its columns

template <class F>
__device__ __forceinline__ void mac4(uint64_t t[4], const uint4& c, uint32_t y) {
  Lazy<F>::mac(t[0], c.x, y);
  Lazy<F>::mac(t[1], c.y, y);
  Lazy<F>::mac(t[2], c.z, y);
  Lazy<F>::mac(t[3], c.w, y);
}

// t += sum_j coef[j] * row[j] over one tile row of cw columns (t folded on return)
template <class F>
__device__ __forceinline__ void lazy_row_tile(uint64_t t[4], const uint32_t* tile_row, const uint4* coef, uint32_t cw) {
  uint32_t j = 0;
  for (; j + 4 <= cw; j += 4) {
    const uint4 y = *reinterpret_cast<const uint4*>(tile_row + j);
    mac4<F>(t, coef[j], y.x);
    mac4<F>(t, coef[j + 1], y.y);
    mac4<F>(t, coef[j + 2], y.z);
    mac4<F>(t, coef[j + 3], y.w);
#pragma unroll
    for (int l = 0; l < 4; l++) t[l] = Lazy<F>::fold(t[l]);
  }
  for (; j < cw; j++) mac4<F>(t, coef[j], tile_row[j]);
#pragma unroll
  for (int l = 0; l < 4; l++) t[l] = Lazy<F>::fold(t[l]);
}

// acc (folded) += a * b in EF4, a given with W*a1..W*a3 (four products per limb)
template <class F>
__device__ __forceinline__ void lazy_ef_mac(uint64_t acc[4], const uint32_t a[4], const uint32_t wa[4], const Ext4& b) {
  using L = Lazy<F>;
#pragma unroll
  for (int l = 0; l < 4; l++) acc[l] = L::fold(acc[l]);
  L::mac(acc[0], a[0], b.c[0]); L::mac(acc[0], wa[1], b.c[3]); L::mac(acc[0], wa[2], b.c[2]); L::mac(acc[0], wa[3], b.c[1]);
  L::mac(acc[1], a[0], b.c[1]); L::mac(acc[1], a[1], b.c[0]); L::mac(acc[1], wa[2], b.c[3]); L::mac(acc[1], wa[3], b.c[2]);
  L::mac(acc[2], a[0], b.c[2]); L::mac(acc[2], a[1], b.c[1]); L::mac(acc[2], a[2], b.c[0]); L::mac(acc[2], wa[3], b.c[3]);
  L::mac(acc[3], a[0], b.c[3]); L::mac(acc[3], a[1], b.c[2]); L::mac(acc[3], a[2], b.c[1]); L::mac(acc[3], a[3], b.c[0]);
}

// Bounds guard of the tile copies: a copy whose shared-memory slot or source
// row/column falls outside its tile or matrix (or a 16-byte copy that is not
// 16-byte aligned) is skipped and the first one recorded; the entry points
// report it after their final synchronisation.
__device__ GuardRecord g_open_guard;
__device__ __noinline__ void open_guard_trip(unsigned long long tag, unsigned long long offset,
                                             unsigned long long extent) {
  if (atomicAdd(&g_open_guard.count, 1ull) == 0) {
    g_open_guard.tag = tag;
    g_open_guard.offset = offset;
    g_open_guard.extent = extent;
    g_open_guard.block = blockIdx.x;
    g_open_guard.thread = threadIdx.x;
  }
}

cudaError_t open_guard_fetch(GuardRecord* dst) { return cudaMemcpyFromSymbol(dst, g_open_guard, sizeof(GuardRecord)); }
cudaError_t open_guard_clear() {
  GuardRecord z{};
  return cudaMemcpyToSymbol(g_open_guard, &z, sizeof z);
}

__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async16(uint32_t* dst, const uint32_t* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Copy tile j0 of matrix M (rows row0 .. row0 + rows - 1, columns j0 .. j0 + 31)
// into `tile` with asynchronous copies; a matrix of at most 32 columns is one
// tile taken as its rows * w contiguous words.
// Tile forms.  A matrix of at most 32 columns is one tile holding its 32 rows:
// with w % 4 == 0 in padded rows (stride kTileStride, 16-byte copies and reads);
// otherwise as the rows * w contiguous words they are in memory (16-byte
// copies when the matrix is 16-byte aligned; lane l reads row l at stride w:
// odd w is conflict-free, w = 2 mod 4 two-way).  Wider matrices: tiles of 32
// columns in padded rows.
__device__ __forceinline__ bool tile_flat(const ReduceMat& M) { return M.w <= 32 && !(M.w % 4 == 0 && M.vec); }

__device__ __forceinline__ void issue_tile(const ReduceMat& M, const uint4* apow, uint32_t apow_len, uint64_t N,
                                           uint64_t row0, uint32_t rows, uint32_t j0, uint32_t* tile, uint32_t lane) {
  const uint32_t w = M.w;
  const uint32_t cw = w <= 32 ? w : min(32u, w - j0);
  const uint32_t* src = M.lde + row0 * w;
  const uint64_t limit = N * w;  // words of the matrix
  // every copy checked: tile slot (data or power part), matrix word, 16-byte alignment
  auto copy = [&](uint32_t dofs, const uint32_t* from, uint64_t from_word, uint64_t from_limit, uint32_t words) {
    if (dofs + words > (uint32_t)kTileBufWords || from_word + words > from_limit) {
      open_guard_trip(kGuardTile, dofs, from_word);
      return;
    }
    if (words == 4) {
      if ((((uintptr_t)(tile + dofs)) | ((uintptr_t)from)) & 15u) {
        open_guard_trip(kGuardLoad, dofs, from_word);
        return;
      }
      cp_async16(tile + dofs, from);
    } else {
      cp_async4(tile + dofs, from);
    }
  };
  // the tile's alpha powers: alpha^(off + j0 + lane) (one point) or alpha^(j0 + lane)
  const uint32_t k0 = (M.multi ? 0u : M.off) + j0;
  if (lane < cw)
    copy(kTileWords + 4 * lane, reinterpret_cast<const uint32_t*>(apow + k0 + lane), 4ull * (k0 + lane),
         4ull * apow_len, 4);
  if (w <= 32) {
    const uint32_t total = rows * w;
    if (!tile_flat(M)) {
      // w % 4 == 0, aligned: padded rows, one 16-byte copy per lane step
      for (uint32_t f = 4 * lane; f < total; f += 4 * 32) {
        const uint32_t r = (uint32_t)(((uint64_t)f * M.magic) >> 32);  // f / w
        copy(r * kTileStride + (f - r * w), src + f, row0 * w + f, limit, 4);
      }
    } else if (M.vec) {
      const uint32_t quads = total >> 2;
      for (uint32_t q = lane; q < quads; q += 32) copy(4 * q, src + 4 * q, row0 * w + 4 * q, limit, 4);
      for (uint32_t f = 4 * quads + lane; f < total; f += 32) copy(f, src + f, row0 * w + f, limit, 1);
    } else {
      for (uint32_t f = lane; f < total; f += 32) copy(f, src + f, row0 * w + f, limit, 1);
    }
    return;
  }
  if (M.vec && w % 4 == 0) {
    // eight lanes per row, four rows per step; cw is a multiple of 4
    const uint32_t rr = lane >> 3, q = (lane & 7) * 4;
    if (q < cw)
      for (uint32_t r = rr; r < rows; r += 4) {
        const uint64_t o = (uint64_t)r * w + j0 + q;
        copy(r * kTileStride + q, src + o, row0 * w + o, limit, 4);
      }
  } else if (lane < cw) {
    for (uint32_t r = 0; r < rows; r++) {
      const uint64_t o = (uint64_t)r * w + j0 + lane;
      copy(r * kTileStride + lane, src + o, row0 * w + o, limit, 1);
    }
  }
}

// t += sum_j coef[j] * row[j], the row at stride 1 but without 16-byte alignment
template <class F>
__device__ __forceinline__ void lazy_row_flat(uint64_t t[4], const uint32_t* tile_row, const uint4* coef, uint32_t cw) {
  uint32_t j = 0;
  for (; j + 4 <= cw; j += 4) {
    const uint32_t y0 = tile_row[j], y1 = tile_row[j + 1], y2 = tile_row[j + 2], y3 = tile_row[j + 3];
    mac4<F>(t, coef[j], y0);
    mac4<F>(t, coef[j + 1], y1);
    mac4<F>(t, coef[j + 2], y2);
    mac4<F>(t, coef[j + 3], y3);
#pragma unroll
    for (int l = 0; l < 4; l++) t[l] = Lazy<F>::fold(t[l]);
  }
  for (; j < cw; j++) mac4<F>(t, coef[j], tile_row[j]);
#pragma unroll
  for (int l = 0; l < 4; l++) t[l] = Lazy<F>::fold(t[l]);
}

// Lane l of a warp owns row row0 + l.  The warp walks the tiles of all
// matrices of the height (32 rows x 32 columns; one tile for a matrix of at
// most 32 columns), double-buffered: the copy of the next tile is in flight
// while the current one is reduced.  Each lane reads its row back across the
// banks; the alpha powers are read by all lanes at the same address.
template <class F, int NS>
__global__ void __launch_bounds__(32 * kReduceWarps, 5) k_reduce(ReduceHeight h) {
  using L = Lazy<F>;
  __shared__ __align__(16) uint32_t tiles[kReduceWarps][2][kTileBufWords];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t N = 1ull << h.log_h;
  const uint64_t row0 = (blockIdx.x * (uint64_t)kReduceWarps + warp) * 32;
  if (row0 >= N || h.n_mats == 0) return;  // whole warp beyond the height
  const uint32_t rows = N - row0 < 32 ? (uint32_t)(N - row0) : 32u;
  const uint64_t i = row0 + lane;
  uint64_t acc[NS][4] = {};
  uint64_t t[4] = {0, 0, 0, 0};
  uint32_t m = 0, j0 = 0, buf = 0;
  ReduceMat M = h.mats[0];
  issue_tile(M, h.apow, h.apow_len, N, row0, rows, 0, tiles[warp][0], lane);
  cp_async_commit();
  for (;;) {
    // the tile after (m, j0)
    uint32_t m2 = m, j2 = j0 + 32;
    if (M.w <= 32 || j2 >= M.w) {
      m2 = m + 1;
      j2 = 0;
    }
    ReduceMat M2;
    if (m2 < h.n_mats) {
      M2 = h.mats[m2];
      issue_tile(M2, h.apow, h.apow_len, N, row0, rows, j2, tiles[warp][buf ^ 1], lane);
    }
    cp_async_commit();
    cp_async_wait_1();
    __syncwarp();
    const uint32_t cw = M.w <= 32 ? M.w : min(32u, M.w - j0);
    const uint4* coef = reinterpret_cast<const uint4*>(tiles[warp][buf] + kTileWords);
    if (tile_flat(M))
      lazy_row_flat<F>(t, tiles[warp][buf] + lane * M.w, coef, cw);
    else
      lazy_row_tile<F>(t, tiles[warp][buf] + lane * kTileStride, coef, cw);
    __syncwarp();  // the buffer is refilled next iteration
    if (m2 != m) {
      // matrix m done
      if (!M.multi) {
#pragma unroll
        for (int q = 0; q < NS; q++)
          if (q == (int)M.slot) {
#pragma unroll
            for (int l = 0; l < 4; l++) acc[q][l] = L::fold(L::fold(acc[q][l]) + t[l]);
          }
      } else {
        // r = sum_j alpha^j M[i][j]; each (slot, alpha^off) term adds alpha^off * r
        Ext4 r;
#pragma unroll
        for (int l = 0; l < 4; l++) r.c[l] = L::finish(t[l]);
        for (uint32_t k = 0; k < M.n_terms; k++) {
          const ReduceTerm T = h.terms[M.term0 + k];
#pragma unroll
          for (int q = 0; q < NS; q++)
            if (q == (int)T.slot) lazy_ef_mac<F>(acc[q], T.a, T.wa, r);
        }
      }
#pragma unroll
      for (int l = 0; l < 4; l++) t[l] = 0;
      if (m2 >= h.n_mats) break;
      M = M2;
    }
    m = m2;
    j0 = j2;
    buf ^= 1;
  }
  if (lane >= rows) return;
  // S_q at this row, stored at its natural position rev(i) (the low coset
  // holds the evaluations at g w_n^rev(i))
  uint32_t* so = h.s_out + bitrev64(i, (int)h.log_h) * h.s_stride + h.s_col0;
#pragma unroll
  for (int q = 0; q < NS; q++) {
    uint4 v;
    v.x = L::finish(acc[q][0]);
    v.y = L::finish(acc[q][1]);
    v.z = L::finish(acc[q][2]);
    v.w = L::finish(acc[q][3]);
    *reinterpret_cast<uint4*>(so + 4 * q) = v;
  }
}

// The reduced opening on the low coset, natural order: for k < 2^log_n,
// ro[k] = sum_q d_q[rev(k)] * (K_q - S_q[k]) (the 1/(z - x) tables are in
// committed, bit-reversed order; S rows of s_stride words, slot q at 4q).
// K_q = S_q(z_q), so every term is a polynomial of degree < n and so is ro:
// its values on the whole LDE domain are its LDE.
template <class F>
__global__ void __launch_bounds__(256) k_reduce_combine(uint32_t log_n, const uint32_t* s, uint32_t s_stride,
                                                        uint32_t n_slots, const uint4* const* dinv, const Ext4* K,
                                                        uint4* ro) {
  using B = Fp<F>;
  using L = Lazy<F>;
  constexpr uint32_t Wm = (uint32_t)((((uint64_t)F::W) << 32) % F::P);
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= (1ull << log_n)) return;
  const uint64_t i = bitrev64(k, (int)log_n);
  uint64_t o[4] = {0, 0, 0, 0};
  for (uint32_t q = 0; q < n_slots; q++) {
    const uint4 sv = __ldg(reinterpret_cast<const uint4*>(s + k * s_stride) + q);
    const Ext4 kq = K[q];
    const Ext4 u{{B::sub(kq.c[0], sv.x), B::sub(kq.c[1], sv.y), B::sub(kq.c[2], sv.z), B::sub(kq.c[3], sv.w)}};
    const Ext4 d = ld4(dinv[q] + i);
    const uint32_t wd[4] = {0, B::mul(d.c[1], Wm), B::mul(d.c[2], Wm), B::mul(d.c[3], Wm)};
    lazy_ef_mac<F>(o, d.c, wd, u);
  }
  Ext4 res;
#pragma unroll
  for (int l = 0; l < 4; l++) res.c[l] = L::finish(o[l]);
  ro[k] = st4(res);
}

cudaError_t launch_reduce_combine(int field, uint32_t log_n, const uint32_t* s, uint32_t s_stride, uint32_t n_slots,
                                  const uint32_t* const* dinv, const uint32_t* K, uint32_t* ro, cudaStream_t st) {
  const uint64_t n = 1ull << log_n;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  auto d = reinterpret_cast<const uint4* const*>(dinv);
  auto k = reinterpret_cast<const Ext4*>(K);
  auto r = reinterpret_cast<uint4*>(ro);
  if (field == 0)
    k_reduce_combine<KoalaBear><<<blocks, 256, 0, st>>>(log_n, s, s_stride, n_slots, d, k, r);
  else
    k_reduce_combine<BabyBear><<<blocks, 256, 0, st>>>(log_n, s, s_stride, n_slots, d, k, r);
  return cudaGetLastError();
}

template <class F>
static cudaError_t launch_reduce_t(const ReduceHeight& h, cudaStream_t st) {
  const uint64_t n = 1ull << h.log_h;
  const unsigned rows_per_block = 32 * kReduceWarps;
  const unsigned blocks = (unsigned)((n + rows_per_block - 1) / rows_per_block);
  const unsigned threads = 32 * kReduceWarps;
  switch (h.n_slots) {
    case 1: k_reduce<F, 1><<<blocks, threads, 0, st>>>(h); break;
    case 2: k_reduce<F, 2><<<blocks, threads, 0, st>>>(h); break;
    case 3: k_reduce<F, 3><<<blocks, threads, 0, st>>>(h); break;
    case 4: k_reduce<F, 4><<<blocks, threads, 0, st>>>(h); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_reduce(int field, const ReduceHeight& h, cudaStream_t st) {
  return field == 0 ? launch_reduce_t<KoalaBear>(h, st) : launch_reduce_t<BabyBear>(h, st);
}

// ---------------------------------------------------------------------------
// Evaluations on a domain: out row k = committed row rev(k) (k < 2^log_d), one
// warp per row, lanes across the columns.
__global__ void k_domain_rows(const uint32_t* lde, uint32_t w, uint32_t log_d, uint32_t* out) {
  const uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (k >= (1ull << log_d)) return;
  const uint32_t* src = lde + bitrev64(k, (int)log_d) * w;
  uint32_t* dst = out + k * w;
  for (uint32_t j = lane; j < w; j += 32) dst[j] = __ldg(src + j);
}

cudaError_t launch_domain_rows(const uint32_t* lde, uint32_t w, uint32_t log_d, uint32_t* out, cudaStream_t st) {
  const uint64_t threads = 32ull << log_d;
  k_domain_rows<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(lde, w, log_d, out);
  return cudaGetLastError();
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
