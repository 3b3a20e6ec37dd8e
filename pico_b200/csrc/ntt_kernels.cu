// Batched coset low-degree extension (Radix2DitParallel::coset_lde_batch
// followed by the row bit-reversal of TwoAdicFriPcs::commit).
//
// Per matrix: evaluations e on H_n (n x w, row-major) -> coefficients
// c = iNTT(e) -> d_i = c_i * g_cb^i for each coset block cb in [0, 2^b) with
// g_cb = shift * w_N^rev_b(cb) -> NTT_n(d) in bit-reversed order.  Output row
// cb*n + j then holds f(shift * w_N^rev_N(cb*n + j)), i.e. committed row i is
// f(shift * w_N^rev(i)) (vm/src/compiler/recursion/circuit/fri.rs:155-171).
//
// Layout: every kernel stages a tile of L rows x LW "lines" in shared memory;
// a line is one column of one sub-transform.  Sub-transforms run as radix-2
// decimation-in-frequency stages (natural in, bit-reversed out) over all
// lines at once; loads and stores walk the row-contiguous dimension fastest so
// that global accesses are coalesced row segments.
//
// One-pass form (n <= 2^11): the whole column tile is resident; read once,
// write once.  Three-pass form, n = n1 * n2 (four-step):
//   A: iNTT_n1 over j1 for each j2, twiddle w_n^-(j2 k1)        -> T1[k1*n2 + j2]
//   B: iNTT_n2 over j2 -> coefficients c[k1 + n1 k2]; per coset: scale,
//      NTT_n2 over k2, twiddle w_n^(k1 k1')                      -> T2[cb*n + k1'*n1 + k1]
//   C: NTT_n1 over k1 -> bit-reversed block                      -> out[cb*n + rev(k1')*n1 + j]
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "field.cuh"
#include "internal.h"

namespace pico {

enum LdePass { kPassSmall = 0, kPassA = 1, kPassB = 2, kPassC = 3 };

// Tiles of one matrix in one pass (host and device).
PICO_HD uint32_t lde_tiles(const LdeMat& m, int pass) {
  if (pass == kPassSmall) return m.log_n1 == 0 ? m.n_ct : 0u;
  if (m.log_n1 == 0) return 0u;
  if (pass == kPassA) return ((1u << m.log_n2) / m.J) * m.n_ct;
  if (pass == kPassB) return ((1u << m.log_n1) / m.J) * m.n_ct;
  return (1u << m.log_b) * ((1u << m.log_n2) / m.J) * m.n_ct;
}

template <class F>
__device__ __forceinline__ uint32_t tw_pow(const TwiddleTables& tw, uint32_t E) {
  return Fp<F>::mul(__ldg(tw.hi + (E >> 14)), __ldg(tw.lo + (E & 0x3fffu)));
}

// w_n^e (or w_n^-e), e in [0, n).
template <class F>
__device__ __forceinline__ uint32_t omega(const TwiddleTables& tw, uint32_t log_n, uint32_t e, bool inv) {
  const uint32_t mask = (1u << F::TWO_ADICITY) - 1u;
  uint32_t E = (e << (F::TWO_ADICITY - log_n)) & mask;
  if (inv) E = (0u - E) & mask;
  return tw_pow<F>(tw, E);
}

// g_cb^i / n from the two-level table of coset cb.
__device__ __forceinline__ const uint32_t* pw_table(const LdeMat& M, uint32_t cb) { return M.pw + cb * 8192u; }
template <class F>
__device__ __forceinline__ uint32_t pw_at(const uint32_t* t, uint32_t i) {
  return Fp<F>::mul(__ldg(t + 4096 + (i >> 12)), __ldg(t + (i & 4095u)));
}

// Matrix owning global tile `tile` of a pass; `local` = tile index within it.
__device__ __forceinline__ const LdeMat& find_tile(const LdeBatch& B, int pass, uint32_t tile, uint32_t& local) {
  uint32_t base = 0, k = 0;
  for (; k + 1 < B.n; k++) {
    const uint32_t t = lde_tiles(B.m[k], pass);
    if (tile < base + t) break;
    base += t;
  }
  local = tile - base;
  return B.m[k];
}

template <class F>
__device__ void fill_twiddles(uint32_t* t, uint32_t log_L, bool inv, const TwiddleTables& tw) {
  const uint32_t h = (1u << log_L) >> 1;
  for (uint32_t i = threadIdx.x; i < h; i += blockDim.x) t[i] = omega<F>(tw, log_L, i, inv);
}

// Radix-2 DIF over L = 2^log_L positions for 2^log_LW lines; tws[t] = w_L^(+-t).
template <class F>
__device__ void smem_dif(uint32_t* buf, uint32_t log_L, uint32_t log_LW, const uint32_t* tws) {
  using B = Fp<F>;
  const uint32_t nb = ((1u << log_L) >> 1) << log_LW;
  for (uint32_t s = 0; s < log_L; s++) {
    const uint32_t log_h = log_L - 1 - s;
    const uint32_t h = 1u << log_h;
    for (uint32_t idx = threadIdx.x; idx < nb; idx += blockDim.x) {
      const uint32_t line = idx & ((1u << log_LW) - 1u);
      const uint32_t b = idx >> log_LW;
      const uint32_t j = b & (h - 1u);
      const uint32_t i0 = ((b >> log_h) << (log_h + 1)) + j;
      uint32_t* p0 = buf + (i0 << log_LW) + line;
      uint32_t* p1 = p0 + (h << log_LW);
      const uint32_t a = *p0, c = *p1;
      *p0 = B::add(a, c);
      *p1 = B::mul(B::sub(a, c), tws[j << s]);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ uint32_t ilog2(uint32_t x) { return 31u - __clz(x); }

// ---------------------------------------------------------------------------
// One-pass form: tile = all n rows of ws columns.
template <class F>
__global__ void __launch_bounds__(256) k_lde_small(const __grid_constant__ LdeBatch batch,
                                                   const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  extern __shared__ uint32_t smem[];
  uint32_t ct;
  const LdeMat& M = find_tile(batch, kPassSmall, blockIdx.x, ct);
  const uint32_t log_L = M.log_n, L = 1u << log_L;
  const uint32_t log_LW = ilog2(M.ws), LW = M.ws;
  const uint32_t w = M.w, col0 = ct * M.ws;
  uint32_t* buf0 = smem;
  uint32_t* buf1 = buf0 + (L << log_LW);
  uint32_t* twf = buf1 + (L << log_LW);
  uint32_t* twi = twf + (L >> 1) + 1;
  fill_twiddles<F>(twf, log_L, false, tw);
  fill_twiddles<F>(twi, log_L, true, tw);
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t c = col0 + (idx & (LW - 1u));
    const uint32_t r = idx >> log_LW;
    buf0[idx] = c < w ? __ldg(M.in + (uint64_t)r * w + c) : 0u;
  }
  __syncthreads();
  smem_dif<F>(buf0, log_L, log_LW, twi);  // position q holds n * c[rev(q)]
  const uint32_t nb = 1u << M.log_b;
  for (uint32_t cb = 0; cb < nb; cb++) {
    const uint32_t* pt = pw_table(M, cb);
    for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
      const uint32_t line = idx & (LW - 1u);
      const uint32_t i = idx >> log_LW;
      buf1[idx] = B::mul(buf0[(bitrev32(i, log_L) << log_LW) + line], pw_at<F>(pt, i));
    }
    __syncthreads();
    smem_dif<F>(buf1, log_L, log_LW, twf);
    uint32_t* outb = M.out + (uint64_t)cb * L * w;
    for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
      const uint32_t c = col0 + (idx & (LW - 1u));
      const uint32_t r = idx >> log_LW;
      if (c < w) outb[(uint64_t)r * w + c] = buf1[idx];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Pass A.
template <class F>
__global__ void __launch_bounds__(256) k_lde_a(const __grid_constant__ LdeBatch batch,
                                               const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassA, blockIdx.x, local);
  const uint32_t log_L = M.log_n1, L = 1u << log_L, log_n2 = M.log_n2;
  const uint32_t log_ws = ilog2(M.ws), ws = M.ws;
  const uint32_t log_LW = log_ws + ilog2(M.J), LW = 1u << log_LW;
  const uint32_t ct = local % M.n_ct, jg = local / M.n_ct;
  const uint32_t j2_0 = jg * M.J, col0 = ct * ws, w = M.w;
  uint32_t* buf = smem;
  uint32_t* twi = buf + (L << log_LW);
  fill_twiddles<F>(twi, log_L, true, tw);
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t line = idx & (LW - 1u);
    const uint32_t m = idx >> log_LW;
    const uint32_t c = col0 + (line & (ws - 1u));
    const uint64_t row = j2_0 + (line >> log_ws) + ((uint64_t)m << log_n2);
    buf[idx] = c < w ? __ldg(M.in + row * w + c) : 0u;
  }
  __syncthreads();
  smem_dif<F>(buf, log_L, log_LW, twi);
  const uint32_t n_mask = (1u << M.log_n) - 1u;
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t line = idx & (LW - 1u);
    const uint32_t k1 = idx >> log_LW;
    const uint32_t c = col0 + (line & (ws - 1u));
    const uint32_t j2 = j2_0 + (line >> log_ws);
    if (c < w) {
      uint32_t v = buf[(bitrev32(k1, log_L) << log_LW) + line];
      v = B::mul(v, omega<F>(tw, M.log_n, (j2 * k1) & n_mask, true));
      M.t1[(((uint64_t)k1 << log_n2) + j2) * w + c] = v;
    }
  }
}

// Pass B.
template <class F>
__global__ void __launch_bounds__(256) k_lde_b(const __grid_constant__ LdeBatch batch,
                                               const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassB, blockIdx.x, local);
  const uint32_t log_L = M.log_n2, L = 1u << log_L, log_n1 = M.log_n1;
  const uint32_t log_ws = ilog2(M.ws), ws = M.ws;
  const uint32_t log_J = ilog2(M.J);
  const uint32_t log_LW = log_ws + log_J, LW = 1u << log_LW;
  const uint32_t ct = local % M.n_ct, kg = local / M.n_ct;
  const uint32_t k1_0 = kg * M.J, col0 = ct * ws, w = M.w;
  const uint64_t n = 1ull << M.log_n;
  uint32_t* buf0 = smem;
  uint32_t* buf1 = buf0 + (L << log_LW);
  uint32_t* twf = buf1 + (L << log_LW);
  uint32_t* twi = twf + (L >> 1) + 1;
  fill_twiddles<F>(twf, log_L, false, tw);
  fill_twiddles<F>(twi, log_L, true, tw);
  // rows k1*n2 + j2: walk c, then j2, then jj
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t cc = idx & (ws - 1u);
    const uint32_t rest = idx >> log_ws;
    const uint32_t j2 = rest & (L - 1u);
    const uint32_t jj = rest >> log_L;
    const uint32_t c = col0 + cc;
    const uint64_t row = ((uint64_t)(k1_0 + jj) << log_L) + j2;
    buf0[(j2 << log_LW) + (jj << log_ws) + cc] = c < w ? __ldg(M.t1 + row * w + c) : 0u;
  }
  __syncthreads();
  smem_dif<F>(buf0, log_L, log_LW, twi);  // position q: n * c[k1 + n1 * rev(q)]
  const uint32_t n_mask = (uint32_t)(n - 1);
  const uint32_t nb = 1u << M.log_b;
  for (uint32_t cb = 0; cb < nb; cb++) {
    const uint32_t* pt = pw_table(M, cb);
    for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
      const uint32_t line = idx & (LW - 1u);
      const uint32_t k2 = idx >> log_LW;
      const uint32_t k1 = k1_0 + (line >> log_ws);
      const uint32_t v = buf0[(bitrev32(k2, log_L) << log_LW) + line];
      buf1[idx] = B::mul(v, pw_at<F>(pt, k1 + (k2 << log_n1)));
    }
    __syncthreads();
    smem_dif<F>(buf1, log_L, log_LW, twf);
    for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
      const uint32_t line = idx & (LW - 1u);
      const uint32_t k1p = idx >> log_LW;
      const uint32_t k1 = k1_0 + (line >> log_ws);
      const uint32_t c = col0 + (line & (ws - 1u));
      if (c < w) {
        uint32_t v = buf1[(bitrev32(k1p, log_L) << log_LW) + line];
        v = B::mul(v, omega<F>(tw, M.log_n, (k1 * k1p) & n_mask, false));
        M.t2[((uint64_t)cb * n + ((uint64_t)k1p << log_n1) + k1) * w + c] = v;
      }
    }
    __syncthreads();
  }
}

// Pass C.
template <class F>
__global__ void __launch_bounds__(256) k_lde_c(const __grid_constant__ LdeBatch batch,
                                               const __grid_constant__ TwiddleTables tw) {
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassC, blockIdx.x, local);
  const uint32_t log_L = M.log_n1, L = 1u << log_L, log_n2 = M.log_n2;
  const uint32_t log_ws = ilog2(M.ws), ws = M.ws;
  const uint32_t log_LW = log_ws + ilog2(M.J);
  const uint32_t groups = (1u << log_n2) / M.J;
  const uint32_t ct = local % M.n_ct;
  const uint32_t rest = local / M.n_ct;
  const uint32_t kg = rest % groups, cb = rest / groups;
  const uint32_t k1p_0 = kg * M.J, col0 = ct * ws, w = M.w;
  const uint64_t n = 1ull << M.log_n;
  uint32_t* buf = smem;
  uint32_t* twf = buf + (L << log_LW);
  fill_twiddles<F>(twf, log_L, false, tw);
  const uint32_t* src = M.t2 + (uint64_t)cb * n * w;
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t cc = idx & (ws - 1u);
    const uint32_t r2 = idx >> log_ws;
    const uint32_t k1 = r2 & (L - 1u);
    const uint32_t jj = r2 >> log_L;
    const uint32_t c = col0 + cc;
    const uint64_t row = ((uint64_t)(k1p_0 + jj) << log_L) + k1;
    buf[(k1 << log_LW) + (jj << log_ws) + cc] = c < w ? __ldg(src + row * w + c) : 0u;
  }
  __syncthreads();
  smem_dif<F>(buf, log_L, log_LW, twf);
  uint32_t* dst = M.out + (uint64_t)cb * n * w;
  for (uint32_t idx = threadIdx.x; idx < (L << log_LW); idx += blockDim.x) {
    const uint32_t cc = idx & (ws - 1u);
    const uint32_t r2 = idx >> log_ws;
    const uint32_t j = r2 & (L - 1u);
    const uint32_t jj = r2 >> log_L;
    const uint32_t c = col0 + cc;
    if (c < w) {
      const uint64_t row = ((uint64_t)bitrev32(k1p_0 + jj, log_n2) << log_L) + j;
      dst[row * w + c] = buf[(j << log_LW) + (jj << log_ws) + cc];
    }
  }
}

// ---------------------------------------------------------------------------
// Power tables of matrix blockIdx.y: for coset cb, entries [0, 4096) hold
// g^e / n and [4096, 8192) hold g^(4096 e), g = shift * w_N^rev_b(cb).
template <class F>
__global__ void k_pow_tables(const __grid_constant__ LdeBatch batch, const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  const LdeMat& M = batch.m[blockIdx.y];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (kPwWords << M.log_b)) return;
  const uint32_t cb = i / kPwWords, e = i % kPwWords;
  const uint32_t log_N = M.log_n + M.log_b;
  const uint32_t g = B::mul(M.shift, omega<F>(tw, log_N, bitrev32(cb, M.log_b), false));
  uint32_t v;
  if (e < 4096u) {
    // 1/2^log_n = p - (p - 1) / 2^log_n (canonical), since 2^log_n * ((p-1)/2^log_n) = -1
    const uint32_t ninv = B::to_monty(F::P - ((F::P - 1u) >> M.log_n));
    v = B::mul(B::pow(g, e), ninv);
  } else {
    v = B::pow(g, (uint64_t)(e - 4096u) << 12);
  }
  M.pw[i] = v;
}

static uint32_t pow2ceil(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

void plan_lde_tiling(LdeMat& m) {
  const uint32_t lw = m.log_n > 22 ? 4u : 8u;  // lines per tile
  m.ws = std::min(lw, pow2ceil(std::max(m.w, 1u)));
  if ((int)m.log_n <= kLdeSmallMaxLog) {
    m.J = 1;
    m.log_n1 = m.log_n2 = 0;
  } else {
    m.J = lw / m.ws;
    m.log_n1 = (m.log_n + 1) / 2;
    m.log_n2 = m.log_n / 2;
  }
  m.n_ct = (m.w + m.ws - 1) / m.ws;
}

static size_t smem_small(const LdeMat& m) {
  const size_t L = 1ull << m.log_n;
  return (2 * L * m.ws + L + 2) * 4;
}
static size_t smem_a(const LdeMat& m) { return ((1ull << m.log_n1) * m.ws * m.J + (1ull << m.log_n1) / 2 + 1) * 4; }
static size_t smem_b(const LdeMat& m) {
  const size_t L = 1ull << m.log_n2;
  return (2 * L * m.ws * m.J + L + 2) * 4;
}
static size_t smem_c(const LdeMat& m) { return smem_a(m); }

template <class F>
static cudaError_t set_smem_attrs() {
  static std::atomic<uint64_t> done_mask{0};  // one bit per device
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0) return e0;
  const uint64_t bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return cudaSuccess;
  const int cap = 227 * 1024;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_lde_small<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  if ((e = cudaFuncSetAttribute(k_lde_a<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  if ((e = cudaFuncSetAttribute(k_lde_b<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  if ((e = cudaFuncSetAttribute(k_lde_c<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  done_mask.fetch_or(bit);
  return cudaSuccess;
}

template <class F>
static cudaError_t launch_lde_t(const LdeMat* mats, uint32_t n_mats, TwiddleTables tw, cudaStream_t st,
                                uint64_t* launches) {
  cudaError_t e = set_smem_attrs<F>();
  if (e) return e;
  for (uint32_t base = 0; base < n_mats; base += kLdeBatch) {
    LdeBatch batch;
    memset(&batch, 0, sizeof batch);
    batch.n = std::min<uint32_t>(kLdeBatch, n_mats - base);
    uint32_t tiles[4] = {0, 0, 0, 0};
    size_t sm[4] = {0, 0, 0, 0};
    uint32_t max_b = 0;
    for (uint32_t k = 0; k < batch.n; k++) {
      const LdeMat& m = mats[base + k];
      batch.m[k] = m;
      max_b = std::max(max_b, m.log_b);
      for (int ps = 0; ps < 4; ps++) tiles[ps] += lde_tiles(m, ps);
      if (lde_tiles(m, kPassSmall)) sm[0] = std::max(sm[0], smem_small(m));
      if (m.log_n1) {
        sm[1] = std::max(sm[1], smem_a(m));
        sm[2] = std::max(sm[2], smem_b(m));
        sm[3] = std::max(sm[3], smem_c(m));
      }
    }
    dim3 pgrid((kPwWords << max_b) / 256, batch.n);
    k_pow_tables<F><<<pgrid, 256, 0, st>>>(batch, tw);
    if ((e = cudaGetLastError())) return e;
    if (launches) *launches += 1;
    if (tiles[kPassSmall]) {
      k_lde_small<F><<<tiles[kPassSmall], 256, sm[0], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      if (launches) *launches += 1;
    }
    if (tiles[kPassA]) {
      k_lde_a<F><<<tiles[kPassA], 256, sm[1], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      k_lde_b<F><<<tiles[kPassB], 256, sm[2], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      k_lde_c<F><<<tiles[kPassC], 256, sm[3], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      if (launches) *launches += 3;
    }
  }
  return cudaSuccess;
}

cudaError_t launch_lde(int field, const LdeMat* mats, uint32_t n_mats, TwiddleTables tw, cudaStream_t st,
                       uint64_t* launches) {
  if (field == 0) return launch_lde_t<KoalaBear>(mats, n_mats, tw, st, launches);
  return launch_lde_t<BabyBear>(mats, n_mats, tw, st, launches);
}

}  // namespace pico
