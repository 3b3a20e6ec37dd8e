// C-ABI implementation: context, device memory accounting, commit planning
// and orchestration, LDE / MMCS / permutation entry points, FRI commit phase.
#include <cuda_runtime.h>
#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "field.cuh"
#include "internal.h"
#include "open.h"
#include "p2_layers.cuh"
#include "runtime.h"
#include "serving.h"

using namespace pico;

namespace pico {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

pico_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PICO_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return PICO_ERR_OUT_OF_MEMORY;
  }
  return PICO_ERR_CUDA;
}

static const uint32_t RC_RAW[30][16] = {
#include "p2_rc_table.inc"
};

template <class F>
static void host_p2_constants(uint32_t ext[8][16], uint32_t inte[24], uint32_t diag[16]) {
  using B = Fp<F>;
  const uint32_t p = F::P;
  for (int r = 0; r < 4; r++)
    for (int j = 0; j < 16; j++) {
      ext[r][j] = B::to_monty(RC_RAW[r][j] % p);
      ext[4 + r][j] = B::to_monty(RC_RAW[4 + F::ROUNDS_P + r][j] % p);
    }
  for (int r = 0; r < F::ROUNDS_P; r++) inte[r] = B::to_monty(RC_RAW[4 + r][0] % p);
  // Internal diagonal (vm/src/primitives/consts.rs:110-154), canonical values.
  uint32_t d[16];
  if (F::ID == 0) {
    const uint32_t k[16] = {p - 2, 1, 2, (p + 1) >> 1, 3, 4, (p - 1) >> 1, p - 3, p - 4,
                            p - ((p - 1) >> 8), p - ((p - 1) >> 3), p - 127, (p - 1) >> 8, (p - 1) >> 3,
                            (p - 1) >> 4, 127};
    memcpy(d, k, sizeof d);
  } else {
    const uint32_t k[16] = {p - 2, 1, 2, (p + 1) >> 1, 3, 4, (p - 1) >> 1, p - 3, p - 4,
                            p - ((p - 1) >> 8), p - ((p - 1) >> 2), p - ((p - 1) >> 3), p - 15, (p - 1) >> 8,
                            (p - 1) >> 4, 15};
    memcpy(d, k, sizeof d);
  }
  for (int j = 0; j < 16; j++) diag[j] = B::to_monty(d[j]);
}

template <class F>
static void host_twiddles(std::vector<uint32_t>& t) {
  using B = Fp<F>;
  t.assign(2 * 16384, 0);
  const uint32_t g = B::to_monty(F::GENERATOR);
  const uint32_t w = B::pow(g, (uint64_t)(F::P - 1) >> F::TWO_ADICITY);
  t[0] = F::ONE;
  for (int j = 1; j < 16384; j++) t[j] = B::mul(t[j - 1], w);
  const uint32_t w14 = B::pow(w, 1ull << 14);
  t[16384] = F::ONE;
  for (int j = 1; j < 16384; j++) t[16384 + j] = B::mul(t[16384 + j - 1], w14);
}

static uint32_t field_two_adicity(int field) { return field == 0 ? 24u : 27u; }

// Host Poseidon2-16 (same round structure and constants as the device
// permutation) for the transcript steps that run on the host: observing the
// opened values and sampling the query indices of TwoAdicFriPcs::open.
template <class F>
struct HostP2 {
  uint32_t ext[8][16], inte[24], diag[16];
  HostP2() { host_p2_constants<F>(ext, inte, diag); }
  // The device permutation's rounds (p2_layers.cuh) with the constants in
  // host memory.
  void permute(uint32_t* s) const {
    using B = Fp<F>;
    p2_external<F>(s);
    for (int r = 0; r < 8; r++) {
      if (r == 4)
        for (int q = 0; q < F::ROUNDS_P; q++) {
          s[0] = p2_sbox<F>(B::add(s[0], inte[q]));
          p2_internal_v2<F>(s, diag);
        }
      for (int j = 0; j < 16; j++) s[j] = p2_sbox<F>(B::add(s[j], ext[r][j]));
      p2_external<F>(s);
    }
  }
};

// The same permutation with the 16-word state in one AVX-512 register (used
// when the host CPU has AVX-512F).  Montgomery products take the even and odd
// lanes through two 32x32->64 multiplies each; the 4x4 external blocks are
// rotations within 128-bit lanes and the cross-block column sums rotations of
// the 128-bit lanes; partial rounds run lane 0's S-box in scalar code while
// the other lanes' diagonal products proceed, then add the lane total.
#define PICO_AVX512 __attribute__((target("avx512f"), always_inline)) inline
template <class F>
struct HostP2Avx512 {
  const HostP2<F>& c;
  explicit HostP2Avx512(const HostP2<F>& consts) : c(consts) {}
  static PICO_AVX512 __m512i add(__m512i a, __m512i b, __m512i p) {
    const __m512i s = _mm512_add_epi32(a, b);
    return _mm512_min_epu32(s, _mm512_sub_epi32(s, p));
  }
  static PICO_AVX512 __m512i mul(__m512i a, __m512i b, __m512i p, __m512i npinv) {
    const __m512i pe = _mm512_mul_epu32(a, b);
    const __m512i po = _mm512_mul_epu32(_mm512_srli_epi64(a, 32), _mm512_srli_epi64(b, 32));
    const __m512i te = _mm512_add_epi64(pe, _mm512_mul_epu32(_mm512_mul_epu32(pe, npinv), p));
    const __m512i to = _mm512_add_epi64(po, _mm512_mul_epu32(_mm512_mul_epu32(po, npinv), p));
    const __m512i r = _mm512_mask_blend_epi32(0xAAAA, _mm512_srli_epi64(te, 32), to);
    return _mm512_min_epu32(r, _mm512_sub_epi32(r, p));
  }
  static PICO_AVX512 __m512i sbox(__m512i x, __m512i p, __m512i npinv) {
    const __m512i x2 = mul(x, x, p, npinv);
    if (F::SBOX == 3) return mul(x2, x, p, npinv);
    return mul(mul(x2, x2, p, npinv), mul(x2, x, p, npinv), p, npinv);
  }
  static PICO_AVX512 __m512i external(__m512i x, __m512i p) {
    const __m512i r1 = _mm512_shuffle_epi32(x, (_MM_PERM_ENUM)0x39);  // lane k <- k+1 within each block
    const __m512i r2 = _mm512_shuffle_epi32(x, (_MM_PERM_ENUM)0x4E);
    const __m512i r3 = _mm512_shuffle_epi32(x, (_MM_PERM_ENUM)0x93);
    const __m512i blk = add(add(x, r1, p), add(r2, r3, p), p);
    // M4 row k: 2 x_k + 3 x_{k+1} + x_{k+2} + x_{k+3} = block sum + x_k + 2 x_{k+1}
    const __m512i m = add(blk, add(x, add(r1, r1, p), p), p);
    const __m512i c1 = _mm512_shuffle_i32x4(m, m, 0x39);
    const __m512i c2 = _mm512_shuffle_i32x4(m, m, 0x4E);
    const __m512i c3 = _mm512_shuffle_i32x4(m, m, 0x93);
    return add(m, add(add(m, c1, p), add(c2, c3, p), p), p);
  }
  // Sum of all 16 lanes, in every lane.
  static PICO_AVX512 __m512i total(__m512i x, __m512i p) {
    __m512i t = add(x, _mm512_shuffle_i32x4(x, x, 0x4E), p);
    t = add(t, _mm512_shuffle_i32x4(t, t, 0xB1), p);
    t = add(t, _mm512_shuffle_epi32(t, (_MM_PERM_ENUM)0x4E), p);
    return add(t, _mm512_shuffle_epi32(t, (_MM_PERM_ENUM)0xB1), p);
  }
  __attribute__((target("avx512f"))) void permute(uint32_t* st) const {
    using B = Fp<F>;
    const __m512i p = _mm512_set1_epi32((int)F::P);
    const __m512i npinv = _mm512_set1_epi32((int)F::NEG_PINV);
    const __m512i diag = _mm512_loadu_si512(c.diag);
    __m512i x = external(_mm512_loadu_si512(st), p);
    for (int r = 0; r < 8; r++) {
      if (r == 4)
        for (int q = 0; q < F::ROUNDS_P; q++) {
          // lanes 1..15 do not depend on lane 0's S-box: their part of the
          // total and their diagonal products run alongside it
          const uint32_t x0 = p2_sbox<F>(B::add((uint32_t)_mm_cvtsi128_si32(_mm512_castsi512_si128(x)), c.inte[q]));
          const __m512i rest = _mm512_mask_set1_epi32(x, 1, 0);
          const __m512i prod = mul(rest, diag, p, npinv);
          const __m512i sum = add(total(rest, p), _mm512_set1_epi32((int)x0), p);
          // lane 0: D_0 = -2
          const uint32_t y0 = B::sub((uint32_t)_mm_cvtsi128_si32(_mm512_castsi512_si128(sum)), B::dbl(x0));
          x = _mm512_mask_set1_epi32(add(prod, sum, p), 1, (int)y0);
        }
      x = sbox(add(x, _mm512_loadu_si512(c.ext[r]), p), p, npinv);
      x = external(x, p);
    }
    _mm512_storeu_si512(st, x);
  }
};
#undef PICO_AVX512

// The AVX2 form: lanes 0-7 in `lo`, 8-15 in `hi` (blocks 0, 1 and 2, 3).
#define PICO_AVX2 __attribute__((target("avx2"), always_inline)) inline
template <class F>
struct HostP2Avx2 {
  const HostP2<F>& c;
  explicit HostP2Avx2(const HostP2<F>& consts) : c(consts) {}
  static PICO_AVX2 __m256i add(__m256i a, __m256i b, __m256i p) {
    const __m256i s = _mm256_add_epi32(a, b);
    return _mm256_min_epu32(s, _mm256_sub_epi32(s, p));
  }
  static PICO_AVX2 __m256i mul(__m256i a, __m256i b, __m256i p, __m256i npinv) {
    const __m256i pe = _mm256_mul_epu32(a, b);
    const __m256i po = _mm256_mul_epu32(_mm256_srli_epi64(a, 32), _mm256_srli_epi64(b, 32));
    const __m256i te = _mm256_add_epi64(pe, _mm256_mul_epu32(_mm256_mul_epu32(pe, npinv), p));
    const __m256i to = _mm256_add_epi64(po, _mm256_mul_epu32(_mm256_mul_epu32(po, npinv), p));
    const __m256i r = _mm256_blend_epi32(_mm256_srli_epi64(te, 32), to, 0xAA);
    return _mm256_min_epu32(r, _mm256_sub_epi32(r, p));
  }
  static PICO_AVX2 __m256i sbox(__m256i x, __m256i p, __m256i npinv) {
    const __m256i x2 = mul(x, x, p, npinv);
    if (F::SBOX == 3) return mul(x2, x, p, npinv);
    return mul(mul(x2, x2, p, npinv), mul(x2, x, p, npinv), p, npinv);
  }
  // M4 on each 4-lane block of one register (block sum + x_k + 2 x_{k+1}).
  static PICO_AVX2 __m256i m4(__m256i x, __m256i p) {
    const __m256i r1 = _mm256_shuffle_epi32(x, 0x39);
    const __m256i blk = add(add(x, r1, p), add(_mm256_shuffle_epi32(x, 0x4E), _mm256_shuffle_epi32(x, 0x93), p), p);
    return add(blk, add(x, add(r1, r1, p), p), p);
  }
  static PICO_AVX2 void external(__m256i& lo, __m256i& hi, __m256i p) {
    lo = m4(lo, p);
    hi = m4(hi, p);
    __m256i col = add(lo, hi, p);
    col = add(col, _mm256_permute2x128_si256(col, col, 0x01), p);
    lo = add(lo, col, p);
    hi = add(hi, col, p);
  }
  static PICO_AVX2 __m256i total(__m256i lo, __m256i hi, __m256i p) {
    __m256i t = add(lo, hi, p);
    t = add(t, _mm256_permute2x128_si256(t, t, 0x01), p);
    t = add(t, _mm256_shuffle_epi32(t, 0x4E), p);
    return add(t, _mm256_shuffle_epi32(t, 0xB1), p);
  }
  __attribute__((target("avx2"))) void permute(uint32_t* st) const {
    using B = Fp<F>;
    const __m256i p = _mm256_set1_epi32((int)F::P);
    const __m256i npinv = _mm256_set1_epi32((int)F::NEG_PINV);
    const __m256i dlo = _mm256_loadu_si256((const __m256i*)c.diag);
    const __m256i dhi = _mm256_loadu_si256((const __m256i*)(c.diag + 8));
    __m256i lo = _mm256_loadu_si256((const __m256i*)st), hi = _mm256_loadu_si256((const __m256i*)(st + 8));
    external(lo, hi, p);
    for (int r = 0; r < 8; r++) {
      if (r == 4)
        for (int q = 0; q < F::ROUNDS_P; q++) {
          const uint32_t x0 = p2_sbox<F>(B::add((uint32_t)_mm_cvtsi128_si32(_mm256_castsi256_si128(lo)), c.inte[q]));
          const __m256i rest = _mm256_blend_epi32(lo, _mm256_setzero_si256(), 0x01);
          const __m256i plo = mul(rest, dlo, p, npinv), phi = mul(hi, dhi, p, npinv);
          const __m256i sum = add(total(rest, hi, p), _mm256_set1_epi32((int)x0), p);
          const uint32_t y0 = B::sub((uint32_t)_mm_cvtsi128_si32(_mm256_castsi256_si128(sum)), B::dbl(x0));
          lo = _mm256_blend_epi32(add(plo, sum, p), _mm256_set1_epi32((int)y0), 0x01);
          hi = add(phi, sum, p);
        }
      lo = sbox(add(lo, _mm256_loadu_si256((const __m256i*)c.ext[r]), p), p, npinv);
      hi = sbox(add(hi, _mm256_loadu_si256((const __m256i*)(c.ext[r] + 8)), p), p, npinv);
      external(lo, hi, p);
    }
    _mm256_storeu_si256((__m256i*)st, lo);
    _mm256_storeu_si256((__m256i*)(st + 8), hi);
  }
};
#undef PICO_AVX2

// Picks the widest form the host CPU runs: PICO_HOST_SIMD=0 forces the scalar
// form, =2 at most AVX2 (for testing the forms against each other).
static int host_simd_level() {
  const char* env = getenv("PICO_HOST_SIMD");
  const int cap = env ? atoi(env) : 3;
  if (cap >= 3 && __builtin_cpu_supports("avx512f")) return 3;
  if (cap >= 2 && __builtin_cpu_supports("avx2")) return 2;
  return 0;
}

void host_permute(int field, uint32_t s[16]) {
  static const HostP2<KoalaBear> kb;
  static const HostP2<BabyBear> bb;
  static const int simd = host_simd_level();
  if (simd == 3) {
    if (field == 0)
      HostP2Avx512<KoalaBear>(kb).permute(s);
    else
      HostP2Avx512<BabyBear>(bb).permute(s);
    return;
  }
  if (simd == 2) {
    if (field == 0)
      HostP2Avx2<KoalaBear>(kb).permute(s);
    else
      HostP2Avx2<BabyBear>(bb).permute(s);
    return;
  }
  if (field == 0)
    kb.permute(s);
  else
    bb.permute(s);
}

// DuplexChallenger<F, Perm, 16, 8> (challenger.rs:89-115).
static void host_duplex(int field, pico_challenger* ch) {
  for (uint32_t i = 0; i < ch->in_len; i++) ch->sponge[i] = ch->in_buf[i];
  ch->in_len = 0;
  host_permute(field, ch->sponge);
  for (int i = 0; i < 8; i++) ch->out_buf[i] = ch->sponge[i];
  ch->out_len = 8;
}
void host_observe(int field, pico_challenger* ch, uint32_t v) {
  ch->out_len = 0;
  ch->in_buf[ch->in_len++] = v;
  if (ch->in_len == 8) host_duplex(field, ch);
}
uint32_t host_sample(int field, pico_challenger* ch) {
  if (ch->in_len != 0 || ch->out_len == 0) host_duplex(field, ch);
  return ch->out_buf[--ch->out_len];
}

}  // namespace pico

// ---------------------------------------------------------------------------
// Context

pico_ctx::~pico_ctx() = default;

// Host-side failure injection for tests (pico_gpu_test_fail_allocations):
// the number of device allocations left before one fails; negative = off.
static std::atomic<int64_t> g_fail_alloc_after{-1};

static pico_status alloc_async(void** p, size_t bytes, cudaStream_t st) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (g_fail_alloc_after.load(std::memory_order_relaxed) >= 0 && g_fail_alloc_after.fetch_sub(1) == 0) {
    set_error("device allocation: injected failure (pico_gpu_test_fail_allocations)");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  return cuda_status(cudaMallocAsync(p, bytes, st), "device allocation");
}

namespace pico {
pico_status device_alloc(void** p, size_t bytes, cudaStream_t st) { return alloc_async(p, bytes, st); }
}  // namespace pico

extern "C" pico_status pico_gpu_test_fail_allocations(int64_t after) {
  g_fail_alloc_after.store(after < 0 ? -1 : after);
  return PICO_OK;
}

static void free_async(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

extern "C" uint32_t pico_gpu_abi_version(void) { return PICO_GPU_ABI_VERSION; }

extern "C" pico_status pico_gpu_challenger_observe(pico_field field, pico_challenger* ch, const uint32_t* values,
                                                   uint64_t n) {
  if (field != PICO_KOALABEAR && field != PICO_BABYBEAR) {
    set_error("challenger_observe: unknown field %d", (int)field);
    return PICO_ERR_INVALID_ARG;
  }
  if (!ch || (n && !values) || ch->in_len > 7 || ch->out_len > 8) {
    set_error("challenger_observe: null argument or corrupt challenger state");
    return PICO_ERR_INVALID_ARG;
  }
  for (uint64_t i = 0; i < n; i++) pico::host_observe(field, ch, values[i]);
  return PICO_OK;
}

extern "C" pico_status pico_gpu_challenger_sample(pico_field field, pico_challenger* ch, uint32_t* out, uint64_t n) {
  if (field != PICO_KOALABEAR && field != PICO_BABYBEAR) {
    set_error("challenger_sample: unknown field %d", (int)field);
    return PICO_ERR_INVALID_ARG;
  }
  if (!ch || (n && !out) || ch->in_len > 7 || ch->out_len > 8) {
    set_error("challenger_sample: null argument or corrupt challenger state");
    return PICO_ERR_INVALID_ARG;
  }
  for (uint64_t i = 0; i < n; i++) out[i] = pico::host_sample(field, ch);
  return PICO_OK;
}
extern "C" const char* pico_gpu_last_error(void) { return g_err.c_str(); }

extern "C" pico_status pico_gpu_init(int device, const pico_config* cfg, pico_ctx** out) {
  if (!out) {
    set_error("pico_gpu_init: null output pointer");
    return PICO_ERR_INVALID_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("pico_gpu_init: no CUDA device");
    return PICO_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("pico_gpu_init: device %d out of range (%d devices)", device, ndev);
    return PICO_ERR_INVALID_ARG;
  }
  pico_status s;
  if ((s = cuda_status(cudaSetDevice(device), "cudaSetDevice"))) return s;
  cudaDeviceProp prop;
  if ((s = cuda_status(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties"))) return s;
  if (prop.major < 10) {
    set_error("pico_gpu_init: device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
              prop.minor);
    return PICO_ERR_UNSUPPORTED;
  }
  auto ctx = std::make_unique<pico_ctx>();
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  // Keep freed memory cached in the device pool instead of returning it.
  cudaMemPool_t pool;
  if ((s = cuda_status(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool"))) return s;
  uint64_t thresh = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh);
  size_t free_b = 0, total_b = 0;
  if ((s = cuda_status(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo"))) return s;
  ctx->budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (uint64_t)(free_b * 0.9);
  const uint32_t ns = (cfg && cfg->n_streams) ? cfg->n_streams : 8;
  ctx->max_inflight = (cfg && cfg->max_inflight) ? std::min(cfg->max_inflight, ns) : ns;
  ctx->max_group = (cfg && cfg->max_group) ? std::min<uint32_t>(cfg->max_group, kMaxGroup) : kDefaultGroup;
  for (uint32_t i = 0; i < ns; i++) {
    cudaStream_t st, cst;
    if ((s = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate"))) return s;
    ctx->streams.push_back(st);
    if ((s = cuda_status(cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking), "cudaStreamCreate"))) return s;
    ctx->copy_streams.push_back(cst);
  }
  for (uint32_t i = 0; i < 4; i++) {
    cudaStream_t st;
    if ((s = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate"))) return s;
    ctx->aux_streams.push_back(st);
  }
  // Constant tables for both fields.
  {
    uint32_t ext[8][16], inte[24] = {0}, diag[16];
    host_p2_constants<KoalaBear>(ext, inte, diag);
    if ((s = cuda_status(upload_p2_constants(0, ext, inte, KoalaBear::ROUNDS_P, diag), "constants"))) return s;
    host_p2_constants<BabyBear>(ext, inte, diag);
    if ((s = cuda_status(upload_p2_constants(1, ext, inte, BabyBear::ROUNDS_P, diag), "constants"))) return s;
  }
  for (int f = 0; f < 2; f++) {
    std::vector<uint32_t> t;
    if (f == 0)
      host_twiddles<KoalaBear>(t);
    else
      host_twiddles<BabyBear>(t);
    void* d = nullptr;
    if ((s = cuda_status(cudaMalloc(&d, (2 * kTwiddleWords + kStageTableWords) * 4), "twiddle tables"))) return s;
    ctx->tw[f] = (uint32_t*)d;
    if ((s = cuda_status(cudaMemcpy(d, t.data(), t.size() * 4, cudaMemcpyHostToDevice), "twiddle upload")))
      return s;
    const TwiddleTables tt = twiddles(ctx.get(), f);
    if ((s = cuda_status(launch_stage_tables(f, tt, const_cast<uint32_t*>(tt.stage), nullptr), "stage tables")) ||
        (s = cuda_status(cudaDeviceSynchronize(), "stage tables")))
      return s;
  }
  {
    void* g = nullptr;
    const size_t bytes = 2 * ctx->streams.size() * sizeof(GuardRecord);
    if ((s = cuda_status(cudaMallocHost(&g, bytes), "guard records"))) return s;
    memset(g, 0, bytes);
    ctx->guard_host = (GuardRecord*)g;
    if ((s = cuda_status(lde_guard_clear(), "guard clear")) || (s = cuda_status(hash_guard_clear(), "guard clear")))
      return s;
  }
  if ((s = serving_start(ctx.get()))) return s;
  *out = ctx.release();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_shutdown(pico_ctx* ctx) {
  if (!ctx) return PICO_OK;
  cudaSetDevice(ctx->device);
  serving_stop(ctx);
  for (auto st : ctx->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto st : ctx->copy_streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto st : ctx->aux_streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (int f = 0; f < 2; f++)
    if (ctx->tw[f]) cudaFree(ctx->tw[f]);
  if (ctx->guard_host) cudaFreeHost(ctx->guard_host);
  delete ctx;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_commit_bytes(pico_field field, const pico_matrix* mats, uint32_t n_mats,
                                             uint32_t log_blowup, uint32_t flags, uint64_t* resident,
                                             uint64_t* scratch) {
  CommitPlan plan;
  pico_status s = plan_commit(field, mats, n_mats, log_blowup, flags, true, plan);
  if (s) return s;
  if (resident) *resident = plan.bytes_resident;
  if (scratch) *scratch = plan.bytes_scratch;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_memory(pico_ctx* ctx, uint64_t* reserved, uint64_t* budget) {
  if (!ctx) {
    set_error("null context");
    return PICO_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> g(ctx->mu);
  if (reserved) *reserved = ctx->reserved;
  if (budget) *budget = ctx->budget;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_reserve_pool(pico_ctx* ctx, uint64_t bytes, uint64_t* pool_bytes) {
  if (!ctx) {
    set_error("reserve_pool: null context");
    return PICO_ERR_INVALID_ARG;
  }
  pico_status s;
  if ((s = cuda_status(cudaSetDevice(ctx->device), "cudaSetDevice"))) return s;
  cudaMemPool_t pool;
  if ((s = cuda_status(cudaDeviceGetDefaultMemPool(&pool, ctx->device), "cudaDeviceGetDefaultMemPool"))) return s;
  bytes = std::min<uint64_t>(bytes, ctx->budget);
  if (bytes) {
    // one allocation of the whole amount, freed at once: the pool keeps it
    // (release threshold unlimited) and splits it for later allocations
    cudaStream_t st = aux_stream(ctx);
    void* p = nullptr;
    if ((s = device_alloc(&p, bytes, st))) return s;
    if ((s = cuda_status(cudaFreeAsync(p, st), "pool reservation"))) return s;
    if ((s = cuda_status(cudaStreamSynchronize(st), "pool reservation"))) return s;
  }
  if (pool_bytes) {
    uint64_t v = 0;  // the attribute is a 64-bit value
    if ((s = cuda_status(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v), "pool size"))) return s;
    *pool_bytes = (uint64_t)v;
  }
  return PICO_OK;
}

namespace pico {

bool try_reserve(pico_ctx* ctx, uint64_t bytes) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->reserved + bytes > ctx->budget) return false;
  ctx->reserved += bytes;
  return true;
}
void unreserve(pico_ctx* ctx, uint64_t bytes) {
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->reserved = bytes > ctx->reserved ? 0 : ctx->reserved - bytes;
  ctx->cv.notify_all();
}
// Streams for read-backs and releases of finished work: they never carry
// long compute, so synchronising them cannot wait on another request.
cudaStream_t aux_stream(pico_ctx* ctx) {
  uint32_t i = ctx->next_aux.fetch_add(1) % (uint32_t)ctx->aux_streams.size();
  return ctx->aux_streams[i];
}

cudaStream_t pick_stream(pico_ctx* ctx, cudaStream_t* copy_stream, uint32_t* slot) {
  uint32_t i = ctx->next_stream.fetch_add(1) % (uint32_t)ctx->streams.size();
  if (copy_stream) *copy_stream = ctx->copy_streams[i];
  if (slot) *slot = i;
  return ctx->streams[i];
}

pico_status guard_enqueue(pico_ctx* ctx, uint32_t slot, cudaStream_t st) {
  pico_status s;
  if ((s = cuda_status(lde_guard_fetch(ctx->guard_host + 2 * slot, st), "guard read-back"))) return s;
  return cuda_status(hash_guard_fetch(ctx->guard_host + 2 * slot + 1, st), "guard read-back");
}

pico_status guard_verdict(pico_ctx* ctx, uint32_t slot, std::string* msg) {
  static const char* const unit[2] = {"LDE", "row hashing"};
  for (int u = 0; u < 2; u++) {
    const GuardRecord& g = ctx->guard_host[2 * slot + u];
    if (!g.count) continue;
    char buf[256];
    snprintf(buf, sizeof buf,
             "internal bounds guard: %s kernel skipped %llu access(es); first: tag %llu, offset %llu of %llu, "
             "block %llu, thread %llu",
             unit[u], g.count, g.tag, g.offset, g.extent, g.block, g.thread);
    if (msg) *msg = buf;
    set_error("%s", buf);
    lde_guard_clear();
    hash_guard_clear();
    memset(ctx->guard_host + 2 * slot, 0, 2 * sizeof(GuardRecord));
    return PICO_ERR_CUDA;
  }
  return PICO_OK;
}
TwiddleTables twiddles(pico_ctx* ctx, int field) {
  TwiddleTables t;
  t.lo = ctx->tw[field];
  t.hi = ctx->tw[field] + kTwiddleWords;
  t.stage = ctx->tw[field] + 2 * kTwiddleWords;
  return t;
}

// ---------------------------------------------------------------------------
// Commit planning

pico_status plan_commit(int field, const pico_matrix* mats, uint32_t n, uint32_t log_b, uint32_t flags, bool extend,
                        CommitPlan& plan, uint32_t shard_log, uint32_t shard) {
  if (field != PICO_KOALABEAR && field != PICO_BABYBEAR) {
    set_error("unknown field %d", field);
    return PICO_ERR_INVALID_ARG;
  }
  if (!mats || n == 0) {
    set_error("commit: no matrices");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t S = field_two_adicity(field);
  if (extend && log_b > kLdeMaxLogBlowup) {
    set_error("commit: log_blowup %u is above the supported %u", log_b, kLdeMaxLogBlowup);
    return PICO_ERR_INVALID_ARG;
  }
  if (shard_log > (extend ? log_b : 0) || (shard_log < 32 && shard >= (1u << shard_log))) {
    set_error("commit: shard %u of 2^%u: a shard must hold whole coset blocks (at most 2^log_blowup = 2^%u shards)",
              shard, shard_log, extend ? log_b : 0);
    return PICO_ERR_INVALID_ARG;
  }
  plan = CommitPlan{};
  plan.field = field;
  plan.log_b = extend ? log_b : 0;
  plan.shard_log = shard_log;
  plan.shard = shard;
  plan.extend = extend;
  plan.input_device = (flags & PICO_INPUT_DEVICE) != 0;
  plan.plain = (flags & PICO_COMMIT_PLAIN) != 0;
  for (uint32_t i = 0; i < n; i++) {
    const pico_matrix& m = mats[i];
    if (m.log_height > 30 || (extend && m.log_height + log_b > S)) {
      set_error("commit: matrix %u height 2^%u with blowup 2^%u exceeds two-adicity %u", i, m.log_height, log_b, S);
      return PICO_ERR_INVALID_ARG;
    }
    if (extend && m.log_height > kLdeMaxLogN) {
      set_error("commit: matrix %u height 2^%u: LDE inputs above 2^%u rows are not supported", i, m.log_height,
                kLdeMaxLogN);
      return PICO_ERR_UNSUPPORTED;
    }
    if (!m.values && m.width) {
      set_error("commit: matrix %u has null values", i);
      return PICO_ERR_INVALID_ARG;
    }
    if (m.flags & ~PICO_MATRIX_EXT4) {
      set_error("commit: matrix %u has unknown flags 0x%x", i, m.flags);
      return PICO_ERR_INVALID_ARG;
    }
    // an extension-field matrix is committed as its base flattening: 4 words per element
    const uint64_t base_w = (uint64_t)m.width * ((m.flags & PICO_MATRIX_EXT4) ? 4u : 1u);
    if (base_w > 0xffffffffull) {
      set_error("commit: matrix %u is too wide", i);
      return PICO_ERR_INVALID_ARG;
    }
    PlannedMat pm;
    pm.input_idx = i;
    pm.log_n = m.log_height;
    pm.log_N = m.log_height + plan.log_b - shard_log;
    pm.w = (uint32_t)base_w;
    pm.shift = m.shift;
    pm.src = m.values;
    plan.mats.push_back(pm);
    plan.cells += base_w << m.log_height;
  }
  std::stable_sort(plan.mats.begin(), plan.mats.end(),
                   [](const PlannedMat& a, const PlannedMat& b) { return a.log_N > b.log_N; });
  plan.log_max = plan.mats[0].log_N;
  for (uint32_t i = 0; i < n;) {
    uint32_t j = i;
    while (j < n && plan.mats[j].log_N == plan.mats[i].log_N) j++;
    plan.groups.push_back({i, j});
    i = j;
  }
  // Memory footprint.
  uint64_t res = 0, scr = 0;
  for (auto& m : plan.mats) {
    const uint64_t cells_in = (uint64_t)m.w << m.log_n;
    const uint64_t cells_out = (uint64_t)m.w << m.log_N;
    if (extend) {
      res += cells_out * 4;
      if (!plan.input_device) scr += cells_in * 4;
      if (m.log_n > (uint32_t)kLdeSmallMaxLog) scr += (cells_in + cells_out) * 4;
      scr += (8192ull << (plan.log_b - shard_log)) * 4 + 64;
    } else if (!plan.input_device) {
      res += cells_in * 4;
    }
  }
  res += ((2ull << plan.log_max) - 1) * 32;
  scr += 4096 + n * (sizeof(LdeMat) + 16);
  // Work counts: one permutation per 8 absorbed elements per row of each
  // height group, one compression per internal node, one more per injected node.
  uint64_t state_rows = 0;  // host inputs: row states of the largest group hashed matrix by matrix
  for (size_t gi = 0; gi < plan.groups.size(); gi++) {
    uint64_t wsum = 0;
    uint32_t nonzero = 0;
    for (uint32_t k = plan.groups[gi].first; k < plan.groups[gi].second; k++) {
      wsum += plan.mats[k].w;
      nonzero += plan.mats[k].w != 0;
      plan.lde_cells += (uint64_t)plan.mats[k].w << plan.mats[k].log_N;
    }
    const uint64_t rows = 1ull << plan.mats[plan.groups[gi].first].log_N;
    if (gi > 0) scr += rows * 32;  // injected-row digests
    // a group hashed matrix by matrix (resumable sponge) keeps row states:
    // host inputs and the plain form, and any group of more matrices with
    // columns than one row-hashing launch takes (kMaxSegs)
    if (nonzero > (uint32_t)kMaxSegs) plan.wide_groups = true;
    if (((!plan.input_device || plan.plain) && nonzero >= 2) || nonzero > (uint32_t)kMaxSegs)
      state_rows = std::max(state_rows, rows);
    const uint64_t absorb = rows * ((wsum + 7) / 8);
    if (gi == 0)
      plan.leaf_permutations = absorb;
    else
      plan.permutations += absorb + rows;
  }
  plan.permutations += plan.leaf_permutations + ((1ull << plan.log_max) - 1);
  scr += state_rows * 64;
  // enqueue_commit carves both blocks into 256-byte aligned sub-buffers
  res += 256ull * (n + 1);
  scr += 256ull * (3ull * n + 4);
  plan.bytes_resident = res;
  plan.bytes_scratch = scr;
  return PICO_OK;
}

// The compression levels of a commit's tree on st: `layers` holds the leaf
// digests; inj[g] (g >= 1) the row digests of height group g, injected at
// the level its height meets.  *root receives the root's address.
pico_status enqueue_tree(const CommitPlan& plan, uint32_t* layers, const std::vector<uint32_t*>& inj,
                         cudaStream_t st, uint64_t* launches, uint32_t** root) {
  pico_status s;
  const int field = plan.field;
  const uint32_t log_max = plan.log_max;
  const uint32_t G = (uint32_t)plan.groups.size();
  uint32_t* layer = layers;
  uint32_t next_group = 1;
  for (uint32_t lvl = 1; lvl <= log_max;) {
    const uint64_t len = 1ull << (log_max - lvl);  // nodes of the level being made
    if (2 * len <= (1u << 15) && 2 * len >= kSubtreeIn) {
      // the narrow levels seven at a time (k_subtree_quad), with the injected
      // rows of the groups whose heights they meet
      SubtreeInj si{};
      for (uint32_t l = 0; l < 7; l++)
        if (next_group < G && plan.mats[plan.groups[next_group].first].log_N == log_max - (lvl + l))
          si.digests[l] = inj[next_group++];
      if ((s = cuda_status(launch_subtree(field, layer, (uint32_t)(2 * len), si, st), "compression"))) return s;
      *launches += 1;
      for (uint32_t l = 0; l < 7; l++) layer += ((2 * len) >> l) * 8;
      lvl += 7;
      continue;
    }
    uint32_t* next = layer + (2 * len) * 8;
    const uint32_t* d = nullptr;
    if (next_group < G && plan.mats[plan.groups[next_group].first].log_N == log_max - lvl) d = inj[next_group++];
    if ((s = cuda_status(launch_compress(field, layer, next, len, d, st), "compression"))) return s;
    *launches += 1;
    layer = next;
    lvl++;
  }
  *root = layer;
  return PICO_OK;
}

// Enqueue a whole commit: LDEs and Poseidon2 on `st`, host -> device input
// copies on `cst`, so copies overlap the compute.  On success `c` holds the
// resident buffers and `scratch` the buffers to free once `st` has passed
// this point (the caller frees them on `st`, which waits for `cst`).
//
// Order of work.  The tree needs every height group's rows: the tallest
// group as leaves, each shorter group as a digest injected at its level.
// Host inputs are copied shortest group first, so the LDEs and row digests
// of the short groups run while the tallest group is still in transit; the
// tallest group's LDE, its leaf hashing and the compression levels come last.
// Matrices of height group gi with columns (width-0 matrices add nothing to a row).
static uint32_t nonzero_mats(const CommitPlan& plan, uint32_t gi) {
  uint32_t c = 0;
  for (uint32_t k = plan.groups[gi].first; k < plan.groups[gi].second; k++) c += plan.mats[k].w != 0;
  return c;
}

// The buffers and descriptors of one commit, made by setup_commit.
struct CommitSetup {
  std::vector<bool> chained;               // per height group: hashed matrix by matrix (resumable sponge)
  std::vector<LdeMat> hm;                  // per planned matrix (extended commits)
  std::vector<const uint32_t*> leaves;     // what the tree hashes, per planned matrix
  std::vector<uint32_t*> inj;              // per height group g >= 1: its row digests
  uint32_t* state = nullptr;               // row states of chained groups
  std::vector<cudaEvent_t> arrived;        // host inputs: matrix k (and all before it) on the device
  CommitSetup() = default;
  CommitSetup(const CommitSetup&) = delete;
  CommitSetup& operator=(const CommitSetup&) = delete;
  ~CommitSetup() {
    for (auto e : arrived)
      if (e) cudaEventDestroy(e);  // released once the device has passed them
  }
};

// Open a commit on st: its events, its device buffers (resident ones into c,
// scratch into `scratch`), the host -> device input copies on cst, and the
// LDE and row-group descriptors over them.
static pico_status setup_commit(pico_ctx* ctx, const CommitPlan& plan, cudaStream_t st, cudaStream_t cst,
                                pico_commit* c, std::vector<void*>& scratch, CommitSetup& cs) {
  pico_status s;
  const int field = plan.field;
  const uint32_t n = (uint32_t)plan.mats.size();
  const uint32_t G = (uint32_t)plan.groups.size();
  const bool copy_in = !plan.input_device;
  c->ctx = ctx;
  c->field = field;
  c->log_max = plan.log_max;
  c->n_mats = n;
  c->shard_log = plan.shard_log;
  c->lde.assign(n, nullptr);
  c->log_N.assign(n, 0);
  c->width.assign(n, 0);
  c->bytes_resident = plan.bytes_resident;
  c->stats.cells = plan.cells;
  c->stats.lde_cells = plan.extend ? plan.lde_cells : 0;
  c->stats.permutations = plan.permutations;
  c->stats.leaf_permutations = plan.leaf_permutations;
  c->stats.lde_bytes = plan.extend ? 4 * (plan.cells + plan.lde_cells) : 0;
  for (int e = 0; e < 7; e++)
    if ((s = cuda_status(cudaEventCreate(&c->ev[e]), "event"))) return s;
  if ((s = cuda_status(cudaEventRecord(c->ev[0], st), "event"))) return s;

  // ---- allocations (stream-ordered on st) ----
  // Resident buffers stay with the commit until release: the LDEs (or, for a
  // commit without extension, the copied host inputs) and the digest layers.
  // Scratch is freed after the commit: host-input staging of extended
  // commits, power tables, four-step scratch, injected-row digests and the
  // chained row states.  A small commit takes each kind as one block carved
  // into 256-byte aligned views: a stream-ordered allocation costs
  // microseconds of host time, and a commit of many small matrices made
  // dozens of them (requests of ~20 matrices of 2^8..2^13 rows went from
  // 1.82 to 1.08 ms).  A large commit allocates each buffer on its own: packed
  // into one block, a 2^30-cell commit's buffers made a later opening of it
  // 10% slower for a 0.5% faster commit.
  std::vector<std::pair<int, size_t>> order;  // (kind, index) in the order buffers are planned
  struct Carve {
    int kind;
    std::vector<std::pair<int, size_t>>* order;
    uint64_t bytes = 0;
    std::vector<uint64_t> off, size;
    std::vector<uint8_t*> ptr;
    uint64_t take(uint64_t b) {
      off.push_back(bytes);
      size.push_back((std::max<uint64_t>(b, 16) + 255) & ~255ull);
      bytes += size.back();
      order->push_back({kind, off.size() - 1});
      return off.size() - 1;
    }
  } res{0, &order}, scr{1, &order};
  constexpr uint64_t kNone = ~0ull;
  constexpr uint64_t kPackedCommitBytes = 256ull << 20;
  // With host inputs, a group of several matrices is hashed one matrix at a
  // time as each arrives (resumable sponge), the row states kept in `state`
  // between matrices; its size is the largest such group's rows x 16 words.
  // The plain form hashes matrix by matrix too (one launch per matrix).
  std::vector<bool>& chained = cs.chained;
  chained.assign(G, false);
  uint64_t rows_max = 0;
  for (uint32_t gi = 0; gi < G; gi++) {
    const uint32_t nz = nonzero_mats(plan, gi);
    chained[gi] = ((copy_in || plan.plain) && nz >= 2) || nz > (uint32_t)kMaxSegs;
    if (chained[gi]) rows_max = std::max<uint64_t>(rows_max, 1ull << plan.mats[plan.groups[gi].first].log_N);
  }
  const uint32_t nb = 1u << (plan.log_b - plan.shard_log);  // coset blocks per LDE
  std::vector<uint64_t> in_bytes(n, 0), ix_in(n, kNone), ix_out(n, kNone), ix_t1(n, kNone), ix_t2(n, kNone);
  for (uint32_t k = 0; k < n; k++) {
    const PlannedMat& m = plan.mats[k];
    in_bytes[k] = ((uint64_t)m.w << m.log_n) * 4;
    if (in_bytes[k] && copy_in) ix_in[k] = plan.extend ? scr.take(in_bytes[k]) : res.take(in_bytes[k]);
  }
  uint64_t ix_pw = kNone;
  if (plan.extend) {
    ix_pw = scr.take((uint64_t)n * nb * kPwWords * 4);
    for (uint32_t k = 0; k < n; k++) {
      const PlannedMat& m = plan.mats[k];
      ix_out[k] = res.take(((uint64_t)m.w << m.log_N) * 4);
      LdeMat probe;
      memset(&probe, 0, sizeof probe);
      probe.log_n = m.log_n;
      plan_lde_tiling(probe, m.log_n <= kLdeMaxLogN ? ctx->lde_split[field][m.log_n] : 0u);
      if (probe.log_n1) {
        ix_t1[k] = scr.take(((uint64_t)m.w << m.log_n) * 4);
        ix_t2[k] = scr.take(((uint64_t)m.w << m.log_N) * 4);
      }
    }
  }
  const uint32_t log_max = plan.log_max;
  const uint64_t ix_layers = res.take(((2ull << log_max) - 1) * 32);
  uint64_t inj_words = 0;
  for (uint32_t g = 1; g < G; g++) inj_words += 8ull << plan.mats[plan.groups[g].first].log_N;
  const uint64_t ix_inj = inj_words ? scr.take(inj_words * 4) : kNone;
  const uint64_t ix_state = rows_max ? scr.take(rows_max * 64) : kNone;
  const char* packed_env = getenv("PICO_PACKED_COMMIT_BYTES");  // tests force either form with it
  const uint64_t packed_max = packed_env ? strtoull(packed_env, nullptr, 10) : kPackedCommitBytes;
  const bool packed = res.bytes + scr.bytes <= packed_max;
  res.ptr.assign(res.off.size(), nullptr);
  scr.ptr.assign(scr.off.size(), nullptr);
  void* d;
  if (packed) {
    for (Carve* cv : {&res, &scr}) {
      if (cv->off.empty()) continue;
      if ((s = alloc_async(&d, cv->bytes, st))) return s;
      (cv == &res ? c->blocks : scratch).push_back(d);
      for (size_t i = 0; i < cv->off.size(); i++) cv->ptr[i] = (uint8_t*)d + cv->off[i];
    }
  }
  // A large commit allocates one buffer at a time, in the order planned; the
  // host-input buffers come first, so the copies start before the rest is
  // allocated.
  size_t allocated = 0;
  auto alloc_through = [&](size_t end) -> pico_status {
    for (; allocated < end; allocated++) {
      const auto& o = order[allocated];
      Carve& cv = o.first == 0 ? res : scr;
      if (pico_status r = alloc_async(&d, cv.size[o.second], st)) return r;
      (o.first == 0 ? c->blocks : scratch).push_back(d);
      cv.ptr[o.second] = (uint8_t*)d;
    }
    return PICO_OK;
  };
  size_t n_inputs = 0;
  for (uint32_t k = 0; k < n; k++) n_inputs += ix_in[k] != kNone;
  if (!packed && (s = alloc_through(n_inputs))) return s;
  auto in_res = [&](uint64_t i) { return (uint32_t*)res.ptr[i]; };
  auto in_scr = [&](uint64_t i) { return (uint32_t*)scr.ptr[i]; };
  std::vector<const uint32_t*> dev_in(n, nullptr);
  for (uint32_t k = 0; k < n; k++) {
    const PlannedMat& m = plan.mats[k];
    if (in_bytes[k] == 0)
      dev_in[k] = nullptr;  // a width-0 matrix: nothing to read, on either side
    else if (!copy_in)
      dev_in[k] = m.src;
    else
      dev_in[k] = plan.extend ? in_scr(ix_in[k]) : in_res(ix_in[k]);
  }

  // ---- host -> device copies on cst: shortest group first, each group's
  // matrices in commit order; arrived[k] marks matrix k (and all before it) ----
  std::vector<cudaEvent_t>& arrived = cs.arrived;
  arrived.assign(n, nullptr);
  if ((s = cuda_status(cudaEventRecord(c->ev[5], st), "event"))) return s;
  if (copy_in) {
    if ((s = cuda_status(cudaStreamWaitEvent(cst, c->ev[5], 0), "copy stream wait"))) return s;
    for (uint32_t gi = G; gi-- > 0;) {
      for (uint32_t k = plan.groups[gi].first; k < plan.groups[gi].second; k++) {
        if (in_bytes[k] &&
            (s = cuda_status(cudaMemcpyAsync(const_cast<uint32_t*>(dev_in[k]), plan.mats[k].src, in_bytes[k],
                                             cudaMemcpyHostToDevice, cst),
                             "input copy")))
          return s;
        cudaEvent_t e;
        if ((s = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))) return s;
        arrived[k] = e;
        if ((s = cuda_status(cudaEventRecord(e, cst), "event"))) return s;
      }
    }
    if ((s = cuda_status(cudaEventRecord(c->ev[6], cst), "event"))) return s;
  } else {
    if ((s = cuda_status(cudaEventRecord(c->ev[6], st), "event"))) return s;
  }

  if (!packed && (s = alloc_through(order.size()))) return s;
  std::vector<LdeMat>& hm = cs.hm;
  hm.assign(plan.extend ? n : 0, LdeMat{});
  std::vector<const uint32_t*>& leaves = cs.leaves;
  leaves.assign(n, nullptr);
  if (plan.extend) {
    uint32_t* pw = in_scr(ix_pw);  // all (matrix, coset) power tables
    for (uint32_t k = 0; k < n; k++) {
      const PlannedMat& m = plan.mats[k];
      LdeMat& L = hm[k];
      memset(&L, 0, sizeof L);
      L.in = dev_in[k];
      L.log_n = m.log_n;
      L.log_b = plan.log_b;
      L.shard_log = plan.shard_log;
      L.shard = plan.shard;
      L.w = m.w;
      L.shift = m.shift % (field == 0 ? KoalaBear::P : BabyBear::P);
      L.pw = pw + (uint64_t)k * nb * kPwWords;
      plan_lde_tiling(L, m.log_n <= kLdeMaxLogN ? ctx->lde_split[field][m.log_n] : 0u);
      L.out = in_res(ix_out[k]);
      c->lde[m.input_idx] = L.out;
      c->log_N[m.input_idx] = m.log_N;
      c->width[m.input_idx] = m.w;
      leaves[k] = L.out;
      if (L.log_n1) {
        if (ix_t1[k] == kNone || ix_t2[k] == kNone) {
          set_error("commit: four-step scratch was not planned for matrix %u", k);
          return PICO_ERR_INVALID_ARG;
        }
        L.t1 = in_scr(ix_t1[k]);
        L.t2 = in_scr(ix_t2[k]);
      }
    }
  } else {
    for (uint32_t k = 0; k < n; k++) {
      const PlannedMat& m = plan.mats[k];
      leaves[k] = dev_in[k];
      c->lde[m.input_idx] = const_cast<uint32_t*>(dev_in[k]);
      c->log_N[m.input_idx] = m.log_N;
      c->width[m.input_idx] = m.w;
    }
  }
  c->layers = in_res(ix_layers);
  // digests of the rows of every shorter height group, injected at its level
  std::vector<uint32_t*>& inj = cs.inj;
  inj.assign(G, nullptr);
  if (inj_words) {
    uint64_t off = 0;
    for (uint32_t g = 1; g < G; g++) {
      inj[g] = in_scr(ix_inj) + off;
      off += 8ull << plan.mats[plan.groups[g].first].log_N;
    }
  }
  cs.state = ix_state == kNone ? nullptr : in_scr(ix_state);
  return PICO_OK;
}

// Phase brackets of a commit's timings (pico_commit::phases) on st.
static pico_status phase_begin(pico_commit* c, int kind, cudaStream_t st) {
  pico_commit::Phase ph;
  ph.kind = kind;
  pico_status r;
  if ((r = cuda_status(cudaEventCreate(&ph.begin), "event"))) return r;
  if ((r = cuda_status(cudaEventCreate(&ph.end), "event"))) {
    cudaEventDestroy(ph.begin);
    return r;
  }
  c->phases.push_back(ph);
  return cuda_status(cudaEventRecord(ph.begin, st), "event");
}
static pico_status phase_end(pico_commit* c, cudaStream_t st) {
  return cuda_status(cudaEventRecord(c->phases.back().end, st), "event");
}

// Row digests of several height groups, gathered into k_hash_groups
// launches of up to kBatchGroups groups and kBatchSegs segments.
struct HashBatcher {
  GroupBatch b;
  HashBatcher() { memset(&b, 0, sizeof b); }
  bool empty() const { return b.n_groups == 0; }
  // Whether the rows of planned matrices [first, last) still fit this launch.
  bool fits(const CommitPlan& plan, uint32_t first, uint32_t last) const {
    uint32_t segs = 0;
    for (uint32_t k = first; k < last; k++) segs += plan.mats[k].w != 0;
    return b.n_groups < (uint32_t)kBatchGroups && b.n_segs + segs <= (uint32_t)kBatchSegs;
  }
  // Add the group of planned matrices [first, last) (rows each, data at
  // leaves[k]); its digests go to out.  Call only when fits().
  void add(const CommitPlan& plan, const std::vector<const uint32_t*>& leaves, uint32_t first, uint32_t last,
           uint64_t rows, uint32_t* out) {
    const uint32_t g = b.n_groups;
    b.seg_begin[g] = b.n_segs;
    uint32_t width = 0;
    for (uint32_t k = first; k < last; k++) {
      if (plan.mats[k].w == 0) continue;
      b.segs[b.n_segs].ptr = leaves[k];
      b.segs[b.n_segs].width = plan.mats[k].w;
      b.n_segs++;
      width += plan.mats[k].w;
    }
    b.seg_begin[g + 1] = b.n_segs;
    b.width[g] = width;
    b.out[g] = out;
    b.row_end[g] = (g ? b.row_end[g - 1] : 0ull) + rows;
    b.n_groups = g + 1;
  }
  pico_status launch(int field, cudaStream_t st, unsigned block) {
    const pico_status r = cuda_status(launch_hash_groups(field, b, st, block), "row hashing");
    memset(&b, 0, sizeof b);
    return r;
  }
};

pico_status enqueue_commit(pico_ctx* ctx, const CommitPlan& plan, cudaStream_t st, cudaStream_t cst,
                           pico_commit* c, std::vector<void*>& scratch, uint32_t* root_host) {
  CommitSetup cs;
  pico_status s = setup_commit(ctx, plan, st, cst, c, scratch, cs);
  if (s) return s;
  const int field = plan.field;
  const uint32_t G = (uint32_t)plan.groups.size();
  const bool copy_in = !plan.input_device;
  const std::vector<bool>& chained = cs.chained;
  const std::vector<LdeMat>& hm = cs.hm;
  const std::vector<const uint32_t*>& leaves = cs.leaves;
  const std::vector<uint32_t*>& inj = cs.inj;
  const std::vector<cudaEvent_t>& arrived = cs.arrived;
  uint32_t* const state = cs.state;

  // ---- compute on st, one height group at a time ----
  // Shortest group first (the order host copies arrive in): its LDE, then
  // the digests of its rows (in the batched form, one launch for all shorter
  // groups, just before the tallest group); the tallest group's rows are the
  // leaves and come last, then the compression levels.  A chained group (host
  // inputs, several matrices) runs matrix by matrix as each arrives: its LDE,
  // then the absorption of its columns into the group's row states.  Each
  // phase sits between a pair of events, so the timings add up exactly.
  const TwiddleTables tw = twiddles(ctx, field);
  // Width-0 matrices add nothing to a row, so they get no segment.
  auto make_group = [&](uint32_t first, uint32_t last, RowGroup& g) {
    memset(&g, 0, sizeof g);
    for (uint32_t k = first; k < last; k++) {
      if (plan.mats[k].w == 0) continue;
      g.segs[g.n_segs].ptr = leaves[k];
      g.segs[g.n_segs].width = plan.mats[k].w;
      g.n_segs++;
      g.total_width += plan.mats[k].w;
    }
  };
  // Width-0 matrices have no LDE work and are left out of the launches.
  auto lde_mats = [&](uint32_t first, uint32_t last) -> pico_status {
    if (!plan.extend) return PICO_OK;
    std::vector<LdeMat> mats;
    for (uint32_t k = first; k < last; k++)
      if (hm[k].w) mats.push_back(hm[k]);
    if (mats.empty()) return PICO_OK;
    if (plan.plain) {
      for (const LdeMat& m : mats)
        if (pico_status r = cuda_status(launch_lde(field, &m, 1, tw, st, &c->stats.launches), "LDE launch"))
          return r;
      return PICO_OK;
    }
    return cuda_status(launch_lde(field, mats.data(), (uint32_t)mats.size(), tw, st, &c->stats.launches),
                       "LDE launch");
  };
  auto begin_phase = [&](int kind) { return phase_begin(c, kind, st); };
  auto end_phase = [&]() { return phase_end(c, st); };
  // The batched form hashes the rows of the shorter groups (those hashed in
  // one pass) together: each is added to `batch` after its LDE, and one
  // launch before the tallest group computes all their digests.  A group
  // with few rows is a few thousand short sponges, latency-bound on its own.
  HashBatcher batch;
  auto flush_batch = [&]() -> pico_status {
    if (batch.empty()) return PICO_OK;
    pico_status r;
    if ((r = begin_phase(pico_commit::kRows))) return r;
    r = batch.launch(field, st, ctx->hash_block[field]);
    c->stats.launches += 1;
    if (!r) r = end_phase();
    return r;
  };
  auto add_to_batch = [&](uint32_t first, uint32_t last, uint64_t rows, uint32_t* out) -> pico_status {
    if (!batch.fits(plan, first, last))
      if (pico_status r = flush_batch()) return r;
    batch.add(plan, leaves, first, last, rows, out);
    return PICO_OK;
  };
  uint32_t* layer = c->layers;
  for (uint32_t gi = G; gi-- > 0 && !s;) {
    const uint32_t first = plan.groups[gi].first, last = plan.groups[gi].second;
    const uint64_t rows = 1ull << plan.mats[first].log_N;
    uint32_t* digests = gi == 0 ? layer : inj[gi];
    const int hash_kind = gi == 0 ? pico_commit::kLeaves : pico_commit::kRows;
    if (gi == 0 && (s = flush_batch())) break;
    if (!chained[gi]) {
      if (copy_in && (s = cuda_status(cudaStreamWaitEvent(st, arrived[last - 1], 0), "wait for inputs"))) break;
      if ((s = begin_phase(pico_commit::kLde)) || (s = lde_mats(first, last)) || (s = end_phase())) break;
      if (gi > 0 && !plan.plain) {
        if ((s = add_to_batch(first, last, rows, digests))) break;
        continue;
      }
      RowGroup g;
      make_group(first, last, g);
      if ((s = begin_phase(hash_kind))) break;
      s = cuda_status(launch_hash_rows(field, g, rows, digests, st, ctx->hash_block[field]),
                      gi == 0 ? "leaf hashing" : "row hashing");
      c->stats.launches += 1;
      if (s || (s = end_phase())) break;
      continue;
    }
    uint32_t cols = 0, left = nonzero_mats(plan, gi);
    for (uint32_t k = first; k < last && !s; k++) {
      if (plan.mats[k].w == 0) continue;
      left--;
      if (copy_in && (s = cuda_status(cudaStreamWaitEvent(st, arrived[k], 0), "wait for inputs"))) break;
      if ((s = begin_phase(pico_commit::kLde)) || (s = lde_mats(k, k + 1)) || (s = end_phase())) break;
      RowGroup g;
      make_group(k, k + 1, g);
      if ((s = begin_phase(hash_kind))) break;
      s = cuda_status(launch_absorb_rows(field, g, rows, cols % 8, cols ? state : nullptr, left ? state : nullptr,
                                         left ? nullptr : digests, st, ctx->hash_block[field]),
                      gi == 0 ? "leaf hashing" : "row hashing");
      c->stats.launches += 1;
      if (s || (s = end_phase())) break;
      cols += plan.mats[k].w;
    }
  }
  if (!s) s = flush_batch();
  if (s) return s;
  if ((s = cuda_status(cudaEventRecord(c->ev[3], st), "event"))) return s;
  if ((s = enqueue_tree(plan, layer, inj, st, &c->stats.launches, &layer))) return s;
  if ((s = cuda_status(cudaEventRecord(c->ev[4], st), "event"))) return s;
  if (root_host)
    if ((s = cuda_status(cudaMemcpyAsync(root_host, layer, 32, cudaMemcpyDeviceToHost, st), "root copy"))) return s;
  return PICO_OK;
}

// Several commits of one field on st, admitted together by the serving
// path: their LDEs share launches (one per pass and sub-transform length for
// every kLdeBatch matrices, shortest traces first so that equal lengths share
// a batch), the rows of all their height groups, the tallest (the leaves)
// included, share k_hash_groups launches, and each commit's compression
// levels follow on their own, its root copied to root_host[i].  Every commit's
// LDE and hashing phases bracket the shared launches, and its launch count
// includes them.  Inputs must be device pointers (no copies to overlap) and
// the commits extended in the batched form.
pico_status enqueue_commit_group(pico_ctx* ctx, const std::vector<const CommitPlan*>& plans, cudaStream_t st,
                                 const std::vector<pico_commit*>& commits, std::vector<void*>& scratch,
                                 const std::vector<uint32_t*>& root_host) {
  const size_t K = plans.size();
  if (K == 0 || commits.size() != K || root_host.size() != K) {
    set_error("commit group: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const int field = plans[0]->field;
  for (const CommitPlan* p : plans)
    if (p->field != field || !p->input_device || !p->extend || p->plain || p->wide_groups) {
      set_error("commit group: members must share the field and be extended batched commits of device inputs "
                "with at most %d matrices of columns per height", kMaxSegs);
      return PICO_ERR_INVALID_ARG;
    }
  pico_status s;
  std::vector<std::unique_ptr<CommitSetup>> cs(K);
  for (size_t i = 0; i < K; i++) {
    cs[i].reset(new CommitSetup());
    if ((s = setup_commit(ctx, *plans[i], st, st, commits[i], scratch, *cs[i]))) return s;
  }
  auto phases = [&](bool begin, int kind) -> pico_status {
    for (size_t i = 0; i < K; i++)
      if (pico_status r = begin ? phase_begin(commits[i], kind, st) : phase_end(commits[i], st)) return r;
    return PICO_OK;
  };
  // LDEs of every member's matrices with columns
  std::vector<LdeMat> lde;
  for (size_t i = 0; i < K; i++)
    for (const LdeMat& m : cs[i]->hm)
      if (m.w) lde.push_back(m);
  std::stable_sort(lde.begin(), lde.end(), [](const LdeMat& a, const LdeMat& b) { return a.log_n < b.log_n; });
  uint64_t shared = 0;
  if ((s = phases(true, pico_commit::kLde))) return s;
  if (!lde.empty() &&
      (s = cuda_status(launch_lde(field, lde.data(), (uint32_t)lde.size(), twiddles(ctx, field), st, &shared),
                       "LDE launch")))
    return s;
  if ((s = phases(false, pico_commit::kLde))) return s;
  // row digests of every height group of every member
  if ((s = phases(true, pico_commit::kLeaves))) return s;
  HashBatcher batch;
  for (size_t i = 0; i < K && !s; i++) {
    const CommitPlan& plan = *plans[i];
    for (uint32_t gi = 0; gi < (uint32_t)plan.groups.size(); gi++) {
      const uint32_t first = plan.groups[gi].first, last = plan.groups[gi].second;
      if (!batch.fits(plan, first, last)) {
        if ((s = batch.launch(field, st, ctx->hash_block[field]))) break;
        shared++;
      }
      batch.add(plan, cs[i]->leaves, first, last, 1ull << plan.mats[first].log_N,
                gi == 0 ? commits[i]->layers : cs[i]->inj[gi]);
    }
  }
  if (!s && !batch.empty()) {
    s = batch.launch(field, st, ctx->hash_block[field]);
    shared++;
  }
  if (s || (s = phases(false, pico_commit::kLeaves))) return s;
  // each member's tree and root
  for (size_t i = 0; i < K; i++) {
    pico_commit* c = commits[i];
    c->stats.launches += shared;
    uint32_t* root = nullptr;
    if ((s = cuda_status(cudaEventRecord(c->ev[3], st), "event"))) return s;
    if ((s = enqueue_tree(*plans[i], c->layers, cs[i]->inj, st, &c->stats.launches, &root))) return s;
    if ((s = cuda_status(cudaEventRecord(c->ev[4], st), "event"))) return s;
    if ((s = cuda_status(cudaMemcpyAsync(root_host[i], root, 32, cudaMemcpyDeviceToHost, st), "root copy")))
      return s;
  }
  return PICO_OK;
}

// Fill c->stats timings from its events (blocks until the commit finished).
// Events: 0 start (st), 3 compression starts (st), 4 root ready (st), 5
// allocations done / copies may start (st), 6 copies done (copy stream); each
// entry of c->phases brackets an LDE, the tallest group's hashing or another
// group's row digests on st.  lde_ms sums the LDE brackets, leaves_ms the
// tallest group's hashing, tree_ms the other groups' row digests plus the
// compression levels.
pico_status finish_stats(pico_commit* c) {
  if (!c->ev[4]) return PICO_OK;
  pico_status s;
  if ((s = cuda_status(cudaEventSynchronize(c->ev[4]), "commit events"))) return s;
  if ((s = cuda_status(cudaEventSynchronize(c->ev[6]), "commit events"))) return s;
  auto span = [&](cudaEvent_t a, cudaEvent_t b, double& acc) -> pico_status {
    float t = 0;
    pico_status r = cuda_status(cudaEventElapsedTime(&t, a, b), "event timing");
    acc += t;
    return r;
  };
  double t_lde = 0, t_leaf = 0, t_tree = 0, t_tot = 0, t_h2d = 0;
  for (const pico_commit::Phase& ph : c->phases) {
    double& acc = ph.kind == pico_commit::kLde ? t_lde : (ph.kind == pico_commit::kLeaves ? t_leaf : t_tree);
    if ((s = span(ph.begin, ph.end, acc))) return s;
  }
  if ((s = span(c->ev[3], c->ev[4], t_tree))) return s;
  if ((s = span(c->ev[0], c->ev[4], t_tot))) return s;
  if ((s = span(c->ev[5], c->ev[6], t_h2d))) return s;
  c->stats.lde_ms = t_lde;
  c->stats.leaves_ms = t_leaf;
  c->stats.tree_ms = t_tree;
  c->stats.h2d_ms = t_h2d;
  c->stats.total_ms = t_tot;
  c->destroy_events();
  return PICO_OK;
}

void free_commit_buffers(pico_commit* c, cudaStream_t st) {
  for (void* b : c->blocks) free_async(b, st);  // LDEs, copied inputs and layers live in these
  c->blocks.clear();
  c->lde.clear();
  c->layers = nullptr;
}

}  // namespace pico

void pico_commit::destroy_events() {
  for (int e = 0; e < 7; e++)
    if (ev[e]) cudaEventDestroy(ev[e]);
  for (const Phase& ph : phases) {
    if (ph.begin) cudaEventDestroy(ph.begin);
    if (ph.end) cudaEventDestroy(ph.end);
  }
  for (cudaEvent_t& e : ev) e = nullptr;
  phases.clear();
}

pico_commit::~pico_commit() { destroy_events(); }

static thread_local pico_commit_stats g_last_stats{};

namespace pico {
// Per-commit and per-request metrics: with PICO_METRICS_LOG set to a path,
// every finished commit (and every served request, with its queue and run
// times) appends one JSON line to that file.  The reference's counterpart is
// its per-chunk proving-time table (vm/src/instances/machine/riscv.rs:255-266).
static std::mutex g_metrics_mu;
void metrics_record(const char* kind, int field, uint32_t n_mats, uint32_t log_b, uint32_t flags,
                    const pico_commit_stats& st, double queued_us, double run_us, uint32_t group) {
  const char* path = getenv("PICO_METRICS_LOG");
  if (!path || !*path) return;
  const double ts = std::chrono::duration<double>(std::chrono::system_clock::now().time_since_epoch()).count();
  char line[768];
  int n = snprintf(line, sizeof line,
                   "{\"ts\": %.6f, \"kind\": \"%s\", \"field\": \"%s\", \"matrices\": %u, \"log_blowup\": %u, "
                   "\"input\": \"%s\", \"form\": \"%s\", \"cells\": %llu, \"lde_cells\": %llu, "
                   "\"permutations\": %llu, \"launches\": %llu, \"total_ms\": %.4f, \"h2d_ms\": %.4f, "
                   "\"lde_ms\": %.4f, \"leaves_ms\": %.4f, \"tree_ms\": %.4f",
                   ts, kind, field == 0 ? "koalabear" : "babybear", n_mats, log_b,
                   (flags & PICO_INPUT_DEVICE) ? "device" : "host", (flags & PICO_COMMIT_PLAIN) ? "plain" : "batched",
                   (unsigned long long)st.cells, (unsigned long long)st.lde_cells,
                   (unsigned long long)st.permutations, (unsigned long long)st.launches, st.total_ms, st.h2d_ms,
                   st.lde_ms, st.leaves_ms, st.tree_ms);
  if (queued_us >= 0 && n > 0 && n < (int)sizeof line)
    n += snprintf(line + n, sizeof line - n, ", \"queued_us\": %.1f, \"run_us\": %.1f, \"group\": %u", queued_us,
                  run_us, group);
  if (n <= 0 || n >= (int)sizeof line - 3) return;
  std::lock_guard<std::mutex> g(g_metrics_mu);
  if (FILE* f = fopen(path, "a")) {
    fprintf(f, "%s}\n", line);
    fclose(f);
  }
}
}  // namespace pico

// ---------------------------------------------------------------------------
// Synchronous commit

static pico_status commit_common(pico_ctx* ctx, pico_field field, const pico_matrix* mats, uint32_t n_mats,
                                 uint32_t log_blowup, uint32_t flags, pico_commit** out, uint32_t root[8],
                                 bool extend, uint32_t shard_log = 0, uint32_t shard = 0) {
  if (!ctx || !root) {
    set_error("commit: null context or root");
    return PICO_ERR_INVALID_ARG;
  }
  if (out) *out = nullptr;
  pico_status s;
  CommitPlan plan;
  if ((s = plan_commit(field, mats, n_mats, log_blowup, flags, extend, plan, shard_log, shard))) return s;
  const uint64_t need = plan.bytes_resident + plan.bytes_scratch;
  if (!try_reserve(ctx, need)) {
    set_error("commit: needs %llu bytes, HBM budget has %llu of %llu reserved", (unsigned long long)need,
              (unsigned long long)ctx->reserved, (unsigned long long)ctx->budget);
    return PICO_ERR_OUT_OF_MEMORY;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t cst;
  uint32_t slot = 0;
  cudaStream_t st = pick_stream(ctx, &cst, &slot);
  auto c = std::make_unique<pico_commit>();
  std::vector<void*> scratch;
  uint32_t root_h[8];
  s = enqueue_commit(ctx, plan, st, cst, c.get(), scratch, root_h);
  // On failure the copy stream may still be writing scratch buffers.
  if (s) cudaStreamSynchronize(cst);
  for (void* p : scratch) cudaFreeAsync(p, st);
  if (!s) s = guard_enqueue(ctx, slot, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "commit");
  if (!s) s = s2;
  if (!s) s = guard_verdict(ctx, slot);
  unreserve(ctx, plan.bytes_scratch);
  if (s) {
    free_commit_buffers(c.get(), st);
    cudaStreamSynchronize(st);
    unreserve(ctx, plan.bytes_resident);
    return s;
  }
  memcpy(c->root, root_h, 32);
  memcpy(root, root_h, 32);
  finish_stats(c.get());
  g_last_stats = c->stats;
  metrics_record(extend ? "commit" : "mmcs_commit", field, n_mats, extend ? log_blowup : 0, flags, c->stats, -1, -1);
  if (out) {
    *out = c.release();
  } else {
    free_commit_buffers(c.get(), st);
    cudaStreamSynchronize(st);
    unreserve(ctx, plan.bytes_resident);
  }
  return PICO_OK;
}

extern "C" pico_status pico_gpu_commit(pico_ctx* ctx, pico_field field, const pico_matrix* mats, uint32_t n_mats,
                                       uint32_t log_blowup, uint32_t flags, pico_commit** out, uint32_t root[8]) {
  return commit_common(ctx, field, mats, n_mats, log_blowup, flags, out, root, true);
}

extern "C" pico_status pico_gpu_mmcs_commit(pico_ctx* ctx, pico_field field, const pico_matrix* mats,
                                            uint32_t n_mats, uint32_t flags, pico_commit** out, uint32_t root[8]) {
  return commit_common(ctx, field, mats, n_mats, 0, flags, out, root, false);
}

extern "C" pico_status pico_gpu_commit_shard(pico_ctx* ctx, pico_field field, const pico_matrix* mats,
                                             uint32_t n_mats, uint32_t log_blowup, uint32_t log_shards,
                                             uint32_t shard, uint32_t flags, pico_commit** out, uint32_t root[8]) {
  return commit_common(ctx, field, mats, n_mats, log_blowup, flags, out, root, true, log_shards, shard);
}

// The tree's top levels over the shard roots: TruncatedPermutation
// compressions, left || right -> the first 8 words of the permuted state.
extern "C" pico_status pico_gpu_merkle_top(pico_field field, const uint32_t* roots, uint32_t log_shards,
                                           uint32_t root[8]) {
  if ((field != PICO_KOALABEAR && field != PICO_BABYBEAR) || !roots || !root || log_shards > 20) {
    set_error("merkle_top: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  std::vector<uint32_t> level(roots, roots + (8ull << log_shards));
  for (uint32_t l = log_shards; l > 0; l--) {
    for (uint64_t i = 0; i < (1ull << (l - 1)); i++) {
      uint32_t s[16];
      memcpy(s, &level[16 * i], 64);
      host_permute(field, s);
      memcpy(&level[8 * i], s, 32);
    }
  }
  memcpy(root, level.data(), 32);
  return PICO_OK;
}

// The siblings of shard s's subtree root on its way up the top levels:
// level k's sibling is root s ^ 1, then the sibling of each parent.
extern "C" pico_status pico_gpu_merkle_top_path(pico_field field, const uint32_t* roots, uint32_t log_shards,
                                                uint32_t shard, uint32_t* path) {
  if ((field != PICO_KOALABEAR && field != PICO_BABYBEAR) || !roots || (log_shards && !path) || log_shards > 20 ||
      shard >= (1u << log_shards)) {
    set_error("merkle_top_path: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  std::vector<uint32_t> level(roots, roots + (8ull << log_shards));
  uint32_t idx = shard;
  for (uint32_t l = log_shards; l > 0; l--) {
    memcpy(path + 8ull * (log_shards - l), &level[8ull * (idx ^ 1)], 32);
    for (uint64_t i = 0; i < (1ull << (l - 1)); i++) {
      uint32_t s[16];
      memcpy(s, &level[16 * i], 64);
      host_permute(field, s);
      memcpy(&level[8 * i], s, 32);
    }
    idx >>= 1;
  }
  return PICO_OK;
}

extern "C" pico_status pico_gpu_commit_stats(const pico_commit* c, pico_commit_stats* out) {
  if (!c || !out) {
    set_error("commit_stats: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  pico_status s = finish_stats(const_cast<pico_commit*>(c));
  if (s) return s;
  *out = c->stats;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_last_commit_stats(pico_commit_stats* out) {
  if (!out) {
    set_error("last_commit_stats: null output");
    return PICO_ERR_INVALID_ARG;
  }
  *out = g_last_stats;
  return PICO_OK;
}

extern "C" pico_status pico_gpu_release(pico_ctx* ctx, pico_commit* c) {
  if (!c) return PICO_OK;
  if (!ctx || c->ctx != ctx) {
    set_error("release: commit belongs to another context");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = aux_stream(ctx);
  free_commit_buffers(c, st);
  pico_status s = cuda_status(cudaStreamSynchronize(st), "release");
  unreserve(ctx, c->bytes_resident);
  delete c;
  return s;
}

extern "C" pico_status pico_gpu_lde_shape(const pico_commit* c, uint32_t mat_idx, uint32_t* log_height,
                                          uint32_t* width) {
  if (!c || mat_idx >= c->n_mats) {
    set_error("lde_shape: bad commit or index");
    return PICO_ERR_INVALID_ARG;
  }
  if (log_height) *log_height = c->log_N[mat_idx];
  if (width) *width = c->width[mat_idx];
  return PICO_OK;
}

extern "C" pico_status pico_gpu_lde_rows(pico_ctx* ctx, const pico_commit* c, uint32_t mat_idx, uint64_t row_begin,
                                         uint64_t row_end, uint32_t* out, uint32_t flags) {
  if (!ctx || !c || !out || mat_idx >= c->n_mats) {
    set_error("lde_rows: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const uint64_t N = 1ull << c->log_N[mat_idx];
  if (row_begin > row_end || row_end > N) {
    set_error("lde_rows: rows [%llu, %llu) outside height %llu", (unsigned long long)row_begin,
              (unsigned long long)row_end, (unsigned long long)N);
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  const uint64_t w = c->width[mat_idx];
  const size_t bytes = (row_end - row_begin) * w * 4;
  if (!bytes) return PICO_OK;
  cudaStream_t st = aux_stream(ctx);
  pico_status s = cuda_status(cudaMemcpyAsync(out, c->lde[mat_idx] + row_begin * w, bytes,
                                              (flags & PICO_OUTPUT_DEVICE) ? cudaMemcpyDeviceToDevice
                                                                           : cudaMemcpyDeviceToHost,
                                              st),
                              "lde_rows copy");
  if (s) return s;
  return cuda_status(cudaStreamSynchronize(st), "lde_rows");
}

extern "C" pico_status pico_gpu_digest_layer(pico_ctx* ctx, const pico_commit* c, uint32_t level, uint32_t* out,
                                             uint32_t flags) {
  if (!ctx || !c || !out || level > c->log_max) {
    set_error("digest_layer: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  uint64_t off = 0;
  for (uint32_t l = 0; l < level; l++) off += 1ull << (c->log_max - l);
  const size_t bytes = (1ull << (c->log_max - level)) * 32;
  cudaStream_t st = aux_stream(ctx);
  pico_status s = cuda_status(
      cudaMemcpyAsync(out, c->layers + off * 8, bytes,
                      (flags & PICO_OUTPUT_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st),
      "digest copy");
  if (s) return s;
  return cuda_status(cudaStreamSynchronize(st), "digest_layer");
}

extern "C" pico_status pico_gpu_open_batch(pico_ctx* ctx, const pico_commit* c, uint64_t index, uint32_t* rows_out,
                                           uint32_t* path_out) {
  if (!ctx || !c || index >= (1ull << c->log_max)) {
    set_error("open_batch: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = aux_stream(ctx);
  pico_status s;
  if (rows_out) {
    uint64_t off = 0;
    for (uint32_t i = 0; i < c->n_mats; i++) {
      const uint64_t r = index >> (c->log_max - c->log_N[i]);
      const uint64_t w = c->width[i];
      if (w) {
        s = cuda_status(cudaMemcpyAsync(rows_out + off, c->lde[i] + r * w, w * 4, cudaMemcpyDeviceToHost, st),
                        "open_batch rows");
        if (s) return s;
      }
      off += w;
    }
  }
  if (path_out) {
    uint64_t off = 0;
    for (uint32_t l = 0; l < c->log_max; l++) {
      const uint64_t sib = (index >> l) ^ 1ull;
      s = cuda_status(cudaMemcpyAsync(path_out + 8 * l, c->layers + (off + sib) * 8, 32, cudaMemcpyDeviceToHost, st),
                      "open_batch path");
      if (s) return s;
      off += 1ull << (c->log_max - l);
    }
  }
  return cuda_status(cudaStreamSynchronize(st), "open_batch");
}

// ---------------------------------------------------------------------------
// Dft / permutation entry points

extern "C" pico_status pico_gpu_coset_lde_batch(pico_ctx* ctx, pico_field field, const uint32_t* in, uint32_t log_n,
                                                uint32_t width, uint32_t log_blowup, uint32_t shift, uint32_t* out,
                                                uint32_t flags) {
  if (!ctx || !in || !out || (field != PICO_KOALABEAR && field != PICO_BABYBEAR)) {
    set_error("coset_lde_batch: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (log_n + log_blowup > field_two_adicity(field)) {
    set_error("coset_lde_batch: 2^%u rows with blowup 2^%u exceeds the two-adicity", log_n, log_blowup);
    return PICO_ERR_INVALID_ARG;
  }
  if (log_n > kLdeMaxLogN) {
    set_error("coset_lde_batch: inputs above 2^%u rows are not supported", kLdeMaxLogN);
    return PICO_ERR_UNSUPPORTED;
  }
  if (flags & PICO_LDE_NATURAL_ORDER) {
    set_error("coset_lde_batch: natural row order is not implemented; the committed order is bit-reversed");
    return PICO_ERR_UNSUPPORTED;
  }
  pico_matrix m{in, log_n, width, shift, 0};
  CommitPlan plan;
  pico_status s;
  if ((s = plan_commit(field, &m, 1, log_blowup, flags, true, plan))) return s;
  const uint64_t out_bytes = ((uint64_t)width << (log_n + log_blowup)) * 4;
  const uint64_t need = plan.bytes_scratch + out_bytes;
  if (!try_reserve(ctx, need)) {
    set_error("coset_lde_batch: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  cudaSetDevice(ctx->device);
  uint32_t slot = 0;
  cudaStream_t st = pick_stream(ctx, nullptr, &slot);
  std::vector<void*> scratch;
  // Reuse the commit planner's LDE path without the tree: build the LdeMat directly.
  LdeMat L;
  memset(&L, 0, sizeof L);
  L.log_n = log_n;
  L.log_b = log_blowup;
  L.w = width;
  plan_lde_tiling(L, ctx->lde_split[field][log_n]);
  const uint64_t in_bytes = ((uint64_t)width << log_n) * 4;
  auto run = [&]() -> pico_status {
    void* p;
    if (flags & PICO_INPUT_DEVICE) {
      L.in = in;
    } else {
      if ((s = alloc_async(&p, in_bytes, st))) return s;
      scratch.push_back(p);
      if ((s = cuda_status(cudaMemcpyAsync(p, in, in_bytes, cudaMemcpyHostToDevice, st), "input copy"))) return s;
      L.in = (const uint32_t*)p;
    }
    if (flags & PICO_OUTPUT_DEVICE) {
      L.out = out;
    } else {
      if ((s = alloc_async(&p, out_bytes, st))) return s;
      scratch.push_back(p);
      L.out = (uint32_t*)p;
    }
    if (L.log_n1) {
      if ((s = alloc_async(&p, in_bytes, st))) return s;
      scratch.push_back(p);
      L.t1 = (uint32_t*)p;
      if ((s = alloc_async(&p, out_bytes, st))) return s;
      scratch.push_back(p);
      L.t2 = (uint32_t*)p;
    }
    const uint32_t nb = 1u << log_blowup;
    if ((s = alloc_async(&p, (uint64_t)nb * kPwWords * 4, st))) return s;
    scratch.push_back(p);
    L.pw = (uint32_t*)p;
    L.shift = shift % (field == 0 ? KoalaBear::P : BabyBear::P);
    if ((s = cuda_status(launch_lde(field, &L, 1, twiddles(ctx, field), st), "LDE"))) return s;
    if (!(flags & PICO_OUTPUT_DEVICE))
      if ((s = cuda_status(cudaMemcpyAsync(out, L.out, out_bytes, cudaMemcpyDeviceToHost, st), "output copy")))
        return s;
    return PICO_OK;
  };
  s = run();
  for (void* p : scratch) cudaFreeAsync(p, st);
  if (!s) s = guard_enqueue(ctx, slot, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "coset_lde_batch");
  if (!s) s = s2;
  if (!s) s = guard_verdict(ctx, slot);
  unreserve(ctx, need);
  return s;
}

extern "C" pico_status pico_gpu_poseidon2_permute(pico_ctx* ctx, pico_field field, uint32_t* states, uint64_t n,
                                                  uint32_t flags) {
  if (!ctx || (!states && n) || (field != PICO_KOALABEAR && field != PICO_BABYBEAR)) {
    set_error("poseidon2_permute: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (!n) return PICO_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t st = pick_stream(ctx);
  pico_status s;
  const uint64_t bytes = n * 64;
  if (flags & PICO_INPUT_DEVICE) {
    if ((s = cuda_status(launch_permute(field, states, n, st, (flags & PICO_P2_FOUR_LANES) != 0), "permute"))) return s;
    return cuda_status(cudaStreamSynchronize(st), "permute");
  }
  if (!try_reserve(ctx, bytes)) {
    set_error("poseidon2_permute: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  void* d;
  s = alloc_async(&d, bytes, st);
  if (!s) s = cuda_status(cudaMemcpyAsync(d, states, bytes, cudaMemcpyHostToDevice, st), "copy in");
  if (!s) s = cuda_status(launch_permute(field, (uint32_t*)d, n, st, (flags & PICO_P2_FOUR_LANES) != 0), "permute");
  if (!s) s = cuda_status(cudaMemcpyAsync(states, d, bytes, cudaMemcpyDeviceToHost, st), "copy out");
  free_async(d, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "permute");
  unreserve(ctx, bytes);
  return s ? s : s2;
}

// ---------------------------------------------------------------------------
// Autotuning

extern "C" pico_status pico_gpu_lde_split(pico_ctx* ctx, pico_field field, uint32_t log_n, uint32_t set_log_n1,
                                          uint32_t* log_n1_out) {
  using namespace pico;
  if (!ctx || (field != PICO_KOALABEAR && field != PICO_BABYBEAR) || log_n > kLdeMaxLogN) {
    set_error("lde_split: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (set_log_n1) {
    if (!lde_split_valid(log_n, set_log_n1)) {
      set_error("lde_split: 2^%u = 2^%u x 2^%u is not a valid split (factors 2^6 .. 2^12, n > 2^11)", log_n,
                set_log_n1, log_n - set_log_n1);
      return PICO_ERR_INVALID_ARG;
    }
    ctx->lde_split[field][log_n] = (uint8_t)set_log_n1;
  }
  if (log_n1_out) {
    LdeMat m;
    memset(&m, 0, sizeof m);
    m.log_n = log_n;
    plan_lde_tiling(m, ctx->lde_split[field][log_n]);
    *log_n1_out = m.log_n1;
  }
  return PICO_OK;
}

// Autotuner cache: with PICO_TUNE_CACHE set to a path, pico_gpu_autotune
// takes the choices recorded there for this device model (name and SM count)
// instead of timing them again, and appends what it times.  One line per
// choice: "<device>|<sms> <field> split <log_n> <log_n1>" or
// "<device>|<sms> <field> hash <block> 0".
namespace {
std::mutex g_tune_mu;
std::string tune_device_key(int device) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "unknown";
  std::string name(prop.name);
  for (char& ch : name)
    if (ch == ' ') ch = '_';
  return name + "|" + std::to_string(prop.multiProcessorCount);
}
struct TuneCache {
  std::map<uint32_t, uint32_t> split;  // log_n -> log_n1
  uint32_t hash_block = 0;
};
TuneCache tune_cache_load(const char* path, const std::string& key, int field) {
  TuneCache c;
  std::lock_guard<std::mutex> g(g_tune_mu);
  FILE* f = fopen(path, "r");
  if (!f) return c;
  char dev[256], kind[16];
  int fld;
  unsigned a, b;
  while (fscanf(f, "%255s %d %15s %u %u", dev, &fld, kind, &a, &b) == 5) {
    if (key != dev || fld != field) continue;
    if (!strcmp(kind, "split") && pico::lde_split_valid(a, b)) c.split[a] = b;
    if (!strcmp(kind, "hash") && (a == 64 || a == 128 || a == 256)) c.hash_block = a;
  }
  fclose(f);
  return c;
}
void tune_cache_append(const char* path, const std::string& key, int field, const std::vector<std::pair<uint32_t, uint32_t>>& splits,
                       uint32_t hash_block) {
  if (splits.empty() && !hash_block) return;
  std::lock_guard<std::mutex> g(g_tune_mu);
  FILE* f = fopen(path, "a");
  if (!f) return;
  for (auto& sp : splits) fprintf(f, "%s %d split %u %u\n", key.c_str(), field, sp.first, sp.second);
  if (hash_block) fprintf(f, "%s %d hash %u 0\n", key.c_str(), field, hash_block);
  fclose(f);
}
}  // namespace

extern "C" pico_status pico_gpu_autotune(pico_ctx* ctx, pico_field field, uint32_t log_n_min, uint32_t log_n_max,
                                         float* ms_out) {
  using namespace pico;
  if (!ctx || (field != PICO_KOALABEAR && field != PICO_BABYBEAR) || log_n_min > log_n_max) {
    set_error("autotune: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const char* cache_path = getenv("PICO_TUNE_CACHE");
  const bool use_cache = cache_path && *cache_path;
  const std::string dev_key = use_cache ? tune_device_key(ctx->device) : std::string();
  const TuneCache cached = use_cache ? tune_cache_load(cache_path, dev_key, field) : TuneCache{};
  std::vector<std::pair<uint32_t, uint32_t>> timed_splits;
  uint32_t timed_block = 0;
  const uint32_t lo = std::max<uint32_t>(log_n_min, kLdeSmallMaxLog + 1);
  const uint32_t hi = std::min<uint32_t>(log_n_max, std::min<uint32_t>(kLdeMaxLogN, field_two_adicity(field) - 1));
  cudaSetDevice(ctx->device);
  uint32_t slot = 0;
  cudaStream_t st = pick_stream(ctx, nullptr, &slot);
  // Synthetic inputs of 2^26 words at most (w = 2^26 / n columns, 4 .. 64),
  // log_blowup 1; the values are zero (timing does not depend on them).
  auto width_for = [](uint32_t log_n) { return std::min<uint32_t>(64, std::max<uint32_t>(4, 1u << (26 - std::min(log_n, 26u)))); };
  uint64_t in_words = 1u << 20, out_words = 2u << 20;
  for (uint32_t l = lo; l <= hi; l++) {
    in_words = std::max<uint64_t>(in_words, (uint64_t)width_for(l) << l);
    out_words = std::max<uint64_t>(out_words, (uint64_t)width_for(l) << (l + 1));
  }
  const uint64_t hash_rows = 1u << 20, hash_w = 64;
  out_words = std::max<uint64_t>(out_words, hash_rows * hash_w);
  const uint64_t need = (2 * in_words + 2 * out_words + 2 * kPwWords + hash_rows * 8) * 4;
  if (!try_reserve(ctx, need)) {
    set_error("autotune: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  std::vector<void*> bufs;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const TwiddleTables tw = twiddles(ctx, field);
  auto run = [&]() -> pico_status {
    pico_status s;
    void *in, *out, *t1, *t2, *pw, *dig;
    if ((s = alloc_async(&in, in_words * 4, st)) || (s = alloc_async(&out, out_words * 4, st)) ||
        (s = alloc_async(&t1, in_words * 4, st)) || (s = alloc_async(&t2, out_words * 4, st)) ||
        (s = alloc_async(&pw, 2 * kPwWords * 4, st)) || (s = alloc_async(&dig, hash_rows * 32, st)))
      return s;
    bufs = {in, out, t1, t2, pw, dig};
    if ((s = cuda_status(cudaMemsetAsync(in, 0, in_words * 4, st), "memset")) ||
        (s = cuda_status(cudaMemsetAsync(out, 0, out_words * 4, st), "memset")) ||
        (s = cuda_status(cudaEventCreate(&e0), "event")) || (s = cuda_status(cudaEventCreate(&e1), "event")))
      return s;
    // time fn over 3 launches after one warm-up; ms per launch
    auto timeit = [&](auto fn, float& ms) -> pico_status {
      pico_status r;
      if ((r = fn())) return r;
      if ((r = cuda_status(cudaEventRecord(e0, st), "event"))) return r;
      for (int i = 0; i < 3; i++)
        if ((r = fn())) return r;
      if ((r = cuda_status(cudaEventRecord(e1, st), "event")) ||
          (r = cuda_status(cudaEventSynchronize(e1), "autotune")) ||
          (r = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "event timing")))
        return r;
      ms /= 3;
      return PICO_OK;
    };
    for (uint32_t l = lo; l <= hi; l++) {
      const uint32_t def = (l + 1) / 2;
      float best = 0;
      uint32_t best_n1 = 0;
      if (auto it = cached.split.find(l); it != cached.split.end()) {
        // from the cache: not timed; the chosen split's time reads -1
        ctx->lde_split[field][l] = (uint8_t)it->second;
        if (ms_out)
          for (int c = 0; c < 3; c++) ms_out[3 * (l - log_n_min) + c] = (def - 1 + c == it->second) ? -1.0f : 0.0f;
        continue;
      }
      for (int c = 0; c < 3; c++) {
        const uint32_t n1 = def - 1 + c;
        float ms = 0;
        if (lde_split_valid(l, n1)) {
          LdeMat m;
          memset(&m, 0, sizeof m);
          m.in = (const uint32_t*)in;
          m.out = (uint32_t*)out;
          m.t1 = (uint32_t*)t1;
          m.t2 = (uint32_t*)t2;
          m.pw = (uint32_t*)pw;
          m.log_n = l;
          m.log_b = 1;
          m.w = width_for(l);
          m.shift = field == 0 ? KoalaBear::ONE : BabyBear::ONE;
          plan_lde_tiling(m, n1);
          if ((s = timeit([&]() { return cuda_status(launch_lde(field, &m, 1, tw, st), "LDE"); }, ms))) return s;
          if (!best_n1 || ms < best) {
            best = ms;
            best_n1 = n1;
          }
        }
        if (ms_out) ms_out[3 * (l - log_n_min) + c] = ms;
      }
      if (best_n1) {
        ctx->lde_split[field][l] = (uint8_t)best_n1;
        timed_splits.push_back({l, best_n1});
      }
    }
    if (cached.hash_block) {
      ctx->hash_block[field] = cached.hash_block;
      if (ms_out)
        for (int c = 0; c < 3; c++) ms_out[3 * (log_n_max - log_n_min + 1) + c] = (64u << c) == cached.hash_block ? -1.0f : 0.0f;
      return PICO_OK;
    }
    RowGroup g;
    memset(&g, 0, sizeof g);
    g.n_segs = 1;
    g.segs[0].ptr = (const uint32_t*)out;
    g.segs[0].width = (uint32_t)hash_w;
    g.total_width = (uint32_t)hash_w;
    float best = 0;
    uint32_t best_block = 256;
    for (int c = 0; c < 3; c++) {
      const unsigned block = 64u << c;
      float ms = 0;
      if ((s = timeit([&]() {
             return cuda_status(launch_hash_rows(field, g, hash_rows, (uint32_t*)dig, st, block), "hash rows");
           }, ms)))
        return s;
      if (c == 0 || ms < best) {
        best = ms;
        best_block = block;
      }
      if (ms_out) ms_out[3 * (log_n_max - log_n_min + 1) + c] = ms;
    }
    ctx->hash_block[field] = best_block;
    timed_block = best_block;
    return PICO_OK;
  };
  pico_status s = run();
  if (!s && use_cache) tune_cache_append(cache_path, dev_key, field, timed_splits, timed_block);
  for (void* p : bufs) cudaFreeAsync(p, st);
  if (!s) s = guard_enqueue(ctx, slot, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "autotune");
  if (!s) s = s2;
  if (!s) s = guard_verdict(ctx, slot);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  unreserve(ctx, need);
  return s;
}
