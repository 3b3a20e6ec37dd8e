// Batched coset low-degree extension (Radix2DitParallel::coset_lde_batch
// followed by the row bit-reversal of TwoAdicFriPcs::commit).
//
// Per matrix: evaluations e on H_n (n x w, row-major) -> coefficients
// c = iNTT(e) -> d_i = c_i * g_cb^i for each coset block cb in [0, 2^b) with
// g_cb = shift * w_N^rev_b(cb) -> NTT_n(d) in bit-reversed order.  Output row
// cb*n + j then holds f(shift * w_N^rev_N(cb*n + j)), i.e. committed row i is
// f(shift * w_N^rev(i)) (vm/src/compiler/recursion/circuit/fri.rs:155-171).
// A shard (LdeMat.shard_log > 0) computes a contiguous range of the blocks:
// every loop over cb below runs over the shard's 2^(b-k) blocks, which sit
// at the start of out, t2 and pw; only the power tables need the global cb.
//
// Tiles.  A CTA of 512 threads stages a tile of L = 2^l positions x LW lines
// in shared memory (L * LW = 2^13 words, 32 KiB plus padding, for l >= 4); a line is one
// column of one sub-transform (J adjacent sub-transforms x ws adjacent
// columns).  The sub-transform length l is a template parameter: one launch
// per (pass, l) group, so every stride, round size and twiddle offset is a
// compile-time constant.  Sub-transforms are decimation-in-frequency (natural
// in, bit-reversed out) and run in rounds of up to four radix-2 stages held in
// registers: a thread loads the 2^r elements a round combines, applies r
// stages and stores them back, so shared memory sees one round trip per four
// stages.  The tile is padded (LW spare words every 16 positions) so that
// neither strided nor stride-1 rounds conflict on banks.
//
// Fusion.  The inverse transform's last round works on 16 consecutive
// positions; those 16 values are exactly the 16 inputs of the forward
// transform's first round (in bit-reversed order), so the coefficients stay
// in registers between the two transforms and are reused for every coset.
// The four-step twiddles and coset scales are geometric along a round's 16
// elements: two table lookups and a running product per set.
//
// One-pass form (n <= 2^11): global -> inverse -> per coset: scale, forward
// -> global.  Three-pass form, n = n1 * n2 (four-step):
//   A: iNTT_n1 over j1 for each j2                              -> T1[k1*n2 + j2]
//   B: times w_n^-(j2 k1), iNTT_n2 over j2 -> coefficients
//      c[k1 + n1 k2]; per coset: scale, NTT_n2 over k2          -> T2[cb*n + k1'*n1 + k1]
//   C: times w_n^(k1 k1'), NTT_n1 over k1 -> bit-reversed block  -> out[cb*n + rev(k1')*n1 + j]
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "field.cuh"
#include "internal.h"

namespace pico {

// Bounds guards.  Every global load and store of these kernels is checked
// against the buffer it belongs to (the pass's input and output, set per CTA
// in s_in / s_out), and every shared-memory and twiddle index against its
// table; an access outside is skipped and the first one is recorded in
// g_lde_guard, which the entry points copy back with their final
// synchronisation and report as an error.  Global accesses are checked once
// per set (its first and last address): checked per element, the guards cost
// 10-17% of the passes' instructions in these issue-bound kernels.
__device__ GuardRecord g_lde_guard;
struct GuardRange {
  const uint32_t* lo;
  const uint32_t* hi;
};
__shared__ GuardRange s_in, s_out;
__shared__ uint32_t s_smem_words;
__device__ __noinline__ void guard_trip(int tag, unsigned long long offset, unsigned long long extent) {
  if (atomicAdd(&g_lde_guard.count, 1ull) == 0) {
    g_lde_guard.tag = tag;
    g_lde_guard.offset = offset;
    g_lde_guard.extent = extent;
    g_lde_guard.block = blockIdx.x;
    g_lde_guard.thread = threadIdx.x;
  }
}
// A set's N accesses p + k * step (k < N) are monotone: checking the first
// and the last covers all of them.
template <int N>
__device__ __forceinline__ bool set_in_range(const uint32_t* p, uint64_t step, const GuardRange& r, int tag) {
  const uint32_t* q = p + (N - 1) * step;
  if (p >= r.lo && q < r.hi) return true;
  guard_trip(tag, (unsigned long long)(p - r.lo), (unsigned long long)(r.hi - r.lo));
  return false;
}

constexpr int kLogTile = 13;   // words per tile for l >= 4: 2^13 (32 KiB)
constexpr int kThreads = 512;  // one 16-element set per thread in a four-stage round
constexpr int kMinLogL3 = 6;   // smallest sub-transform of the three-pass form (n = 2^12)
constexpr int kMaxLogL = 12;   // largest sub-transform (n <= 2^24)

enum LdePass { kPassSmall = 0, kPassA = 1, kPassB = 2, kPassC = 3 };

PICO_HD uint32_t ceil_log2(uint32_t x) {
  uint32_t l = 0;
  while ((1u << l) < x) l++;
  return l;
}

// Lines per tile (log2) at sub-transform length 2^l: 2^13 words for l >= 4;
// below that, 512 lines (a single round of 2^l positions per thread).
PICO_HD constexpr uint32_t tile_log_lw(uint32_t l) {
  return l < 4 ? 9u : (l >= (uint32_t)kLogTile ? 0u : (uint32_t)kLogTile - l);
}

constexpr int rev_bits(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

struct PassGeom {
  uint32_t log_L, log_other, log_ws, log_J, n_ct, groups;
};

// Tile geometry of a pass: sub-transform length 2^log_L, 2^log_other
// sub-transforms side by side.  A tile's LW lines split into ws columns
// times J adjacent sub-transforms; in the three-pass form ws is at most 64
// (256 bytes of a row).  Lines past the matrix (columns >= w, or
// sub-transforms >= 2^log_other) are inactive.
PICO_HD PassGeom pass_geom(const LdeMat& m, int pass) {
  PassGeom g;
  if (pass == kPassSmall) {
    g.log_L = m.log_n;
    g.log_other = 0;
  } else if (pass == kPassB) {
    g.log_L = m.log_n2;
    g.log_other = m.log_n1;
  } else {
    g.log_L = m.log_n1;
    g.log_other = m.log_n2;
  }
  const uint32_t log_LW = tile_log_lw(g.log_L);
  const uint32_t cw = ceil_log2(m.w > 0 ? m.w : 1u);
  g.log_ws = cw < log_LW ? cw : log_LW;
  if (pass != kPassSmall && g.log_ws > 6) g.log_ws = 6;
  g.log_J = log_LW - g.log_ws;
  g.n_ct = (m.w + (1u << g.log_ws) - 1) >> g.log_ws;
  g.groups = g.log_J >= g.log_other ? 1u : 1u << (g.log_other - g.log_J);
  return g;
}

// Tiles of one matrix in one pass (host and device).
PICO_HD uint32_t lde_tiles(const LdeMat& m, int pass) {
  if ((pass == kPassSmall) != (m.log_n1 == 0)) return 0u;
  const PassGeom g = pass_geom(m, pass);
  const uint32_t t = g.groups * g.n_ct;
  return pass == kPassC ? t << lde_log_c(m) : t;
}

PICO_HD uint32_t pass_log_L(const LdeMat& m, int pass) {
  return pass == kPassSmall ? m.log_n : (pass == kPassB ? m.log_n2 : m.log_n1);
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
__device__ __forceinline__ const uint32_t* pw_table(const LdeMat& M, uint32_t cb) { return M.pw + cb * kPwWords; }
template <class F>
__device__ __forceinline__ uint32_t pw_at(const uint32_t* t, uint32_t i) {
  if (i >= (1u << 24)) { guard_trip(kGuardPowIndex, i, 1u << 24); i = 0; }
  return Fp<F>::mul(__ldg(t + 4096 + (i >> 12)), __ldg(t + (i & 4095u)));
}

// n = 2^log_n in Monty form.
template <class F>
__device__ __forceinline__ uint32_t n_monty(uint32_t log_n) {
  return Fp<F>::to_monty(1u << log_n);
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

// Twiddles of a 2^LOG_L-point transform in shared memory, one table per
// stage: stage s holds w_L^(+-(x << s)) for x < L >> (s+1) at entry
// L - (L >> s) (L - 1 entries in all).  An entry is the pair {w, w'}: w the
// twiddle's canonical value and w' = floor(w * 2^32 / p), Shoup's
// precomputed quotient, so a butterfly multiplies by it without a
// Montgomery reduction (bfly below).  A round's threads read consecutive x,
// which sit on distinct banks.  The exception is the fused first forward
// round, whose x differ in bits 4 .. l-5 (x = rev(q) + c * L/16); for
// l >= 9 (fewer than 32 lines) the tables of stages 0..3 therefore store
// entry x at x ^ ((x >> 4) & (2^(l-8) - 1)).  Every access to those tables
// has x = o + c * L/16 with o < L/16, so the swizzle applies to o alone.
// The tables of every length are built once per context (k_stage_tables:
// forward then inverse, 2^l entries each, lengths 2^1 .. 2^12 back to back
// from entry 2^(l+1) - 4) and each CTA copies the two it needs.
template <int LOG_L>
__device__ __forceinline__ constexpr uint32_t tw_off(int s) {
  return (1u << LOG_L) - ((1u << LOG_L) >> s);
}
PICO_HD uint32_t tw_swz_l(uint32_t l, uint32_t x) { return l >= 9 ? x ^ ((x >> 4) & ((1u << (l - 8)) - 1u)) : x; }
template <int LOG_L>
__device__ __forceinline__ uint32_t tw_swz(uint32_t x) {
  return tw_swz_l(LOG_L, x);
}
PICO_HD constexpr uint32_t stage_base(uint32_t l) { return (2u << l) - 4u; }
static_assert(2 * stage_base(13) <= kStageTableWords, "stage tables fit");

// Copy one direction's tables (2^LOG_L entries of two words) to shared memory.
template <int LOG_L>
__device__ __forceinline__ void load_twiddles(uint32_t* dst, const TwiddleTables& tw, bool inv) {
  const uint32_t* src = tw.stage + 2 * (stage_base(LOG_L) + (inv ? (1u << LOG_L) : 0u));
  if constexpr (LOG_L >= 1) {
    for (uint32_t i = threadIdx.x; i < (1u << LOG_L) / 2; i += kThreads)
      reinterpret_cast<uint4*>(dst)[i] = __ldg(reinterpret_cast<const uint4*>(src) + i);
  } else {
    if (threadIdx.x < 2) dst[threadIdx.x] = __ldg(src + threadIdx.x);
  }
}

// One entry of the stage tables: length 2^l (l = 1..12), direction, stage s,
// entry x at its swizzled position; the last entry of each table is unused.
template <class F>
__global__ void k_stage_tables(const __grid_constant__ TwiddleTables tw, uint32_t* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= stage_base(kMaxLogL + 1)) return;
  uint32_t l = 1;
  while (stage_base(l + 1) <= i) l++;
  const uint32_t L = 1u << l;
  uint32_t r = i - stage_base(l);
  const bool inv = r >= L;
  if (inv) r -= L;
  uint32_t v = 0;
  if (r < L - 1) {
    uint32_t s = 0;
    while (r >= L - (L >> (s + 1))) s++;
    uint32_t x = r - (L - (L >> s));
    if (s < 4) x = tw_swz_l(l, x);  // the swizzle is its own inverse
    v = omega<F>(tw, l, x << s, inv);
  }
  // Monty(a) * w for canonical w is Monty(a * w): the butterflies multiply
  // by the canonical value
  const uint32_t c = Fp<F>::from_monty(v);
  out[2 * i] = c;
  out[2 * i + 1] = (uint32_t)(((uint64_t)c << 32) / F::P);
}

// Shared-memory layout of a tile: position-major, LW lines per position.
// With fewer than 32 lines, LW spare words follow every 16 positions (word
// (pos + pos/16) * LW + line), which puts every warp access of every round
// below on distinct banks; with 32 or more lines the lines alone do.  Within
// a set of a round the positions are base + k * stride with stride a multiple
// of 16, or stride 1 from a base aligned to the set, so the padded words are
// row + k * step: one address computation per set, the rest immediates.
PICO_HD constexpr uint32_t tile_words_l(uint32_t l) {
  return ((1u << l) + (tile_log_lw(l) < 5 ? (1u << l) >> 4 : 0u)) << tile_log_lw(l);
}
template <int LOG_LW>
__device__ __forceinline__ uint32_t srow(uint32_t pos, uint32_t line) {
  if constexpr (LOG_LW >= 5) {
    return (pos << LOG_LW) + line;
  } else {
    return ((pos + (pos >> 4)) << LOG_LW) + line;
  }
}
template <int LOG_LW, int LOG_STRIDE>
__device__ __forceinline__ constexpr uint32_t sstep() {
  return (LOG_LW >= 5 || LOG_STRIDE < 4 ? (1u << LOG_STRIDE) : (1u << LOG_STRIDE) + (1u << (LOG_STRIDE - 4)))
         << LOG_LW;
}
// Row of a set of N elements; the guard checks the set's last word.
template <int LOG_LW, int LOG_STRIDE, int N>
__device__ __forceinline__ uint32_t set_row(uint32_t pos, uint32_t line) {
  uint32_t r = srow<LOG_LW>(pos, line);
  if (r + (uint32_t)(N - 1) * sstep<LOG_LW, LOG_STRIDE>() >= s_smem_words) {
    guard_trip(kGuardTile, r, s_smem_words);
    r = 0;
  }
  return r;
}

// DIF butterfly: (a, b) -> (a + b, (a - b) * w), canonical in and out.
// The product is Shoup's: with w' = floor(w * 2^32 / p) and q the high word
// of d * w', d * w - q * p lies in [0, 2p) for every 32-bit d (here
// d = a - b + p < 2p), computed in 32-bit arithmetic; one conditional
// subtraction makes it canonical.  Two 32-bit multiplies and one high
// multiply, against the two wide multiplies and one low multiply of a
// Montgomery product: 1.5x the butterflies per clock on this part.
template <class F>
__device__ __forceinline__ void bfly(uint32_t& a, uint32_t& b, uint2 w) {
  using B = Fp<F>;
  const uint32_t x = B::add(a, b);
  const uint32_t d = a - b + F::P;
  const uint32_t q = __umulhi(d, w.y);
  b = B::canon(d * w.x - q * F::P);
  a = x;
}

// Stages S0 .. S0+R-1 of a 2^LOG_L-point DIF on v[k] = x[base + k * stride],
// stride = L >> (S0 + R), base = blk * (L >> S0) + o;  tw = the per-stage
// tables above.  The twiddle of stage s at position x is
// w_L^((x mod (L >> (s+1))) << s), and x mod (L >> (s+1)) = o + (k mod half) * stride.
template <class F, int LOG_L, int S0, int R>
__device__ __forceinline__ void dif(uint32_t* v, uint32_t o, const uint32_t* tw) {
  constexpr int N = 1 << R;
  constexpr uint32_t stride = 1u << (LOG_L - S0 - R);
  static_assert(S0 == 0 || S0 >= 4 || LOG_L < 9, "swizzled stage tables are read by first rounds only");
  const uint32_t o_sw = S0 == 0 ? tw_swz<LOG_L>(o) : o;
#pragma unroll
  for (int t = 0; t < R; t++) {
    const int half = N >> (t + 1);
#pragma unroll
    for (int k = 0; k < N; k++) {
      if (k & half) continue;
      // in range by construction: o < stride (RoundGeo masks it; the
      // swizzle only permutes o's bits below stride), so the entry
      // o + (k mod half) * stride < stride * half = L >> (s+1) lies inside
      // stage s's table, which ends at tw_off(s) + (L >> (s+1)) < L
      const uint32_t ti = o_sw + tw_off<LOG_L>(S0 + t) + (uint32_t)(k & (half - 1)) * stride;
      bfly<F>(v[k], v[k + half], reinterpret_cast<const uint2*>(tw)[ti]);
    }
  }
}

// Work items of a round (S0, R): 2^(LOG_L - R) sets per line.  Item `it` ->
// its line, offset o within the stride and first position.
template <int LOG_L, int S0, int R>
struct RoundGeo {
  static constexpr int LOG_LW = (int)tile_log_lw(LOG_L);
  static constexpr int LOG_STRIDE = LOG_L - S0 - R;
  static constexpr int N_ITEMS = 1 << (LOG_L - R + LOG_LW);
  static constexpr int PER_THREAD = N_ITEMS >= kThreads ? N_ITEMS / kThreads : 1;
  static_assert(N_ITEMS % kThreads == 0, "rounds cover whole thread blocks");
  static __device__ __forceinline__ void item(uint32_t it, uint32_t& line, uint32_t& o, uint32_t& base) {
    line = it & ((1u << LOG_LW) - 1u);
    const uint32_t q = it >> LOG_LW;
    o = q & ((1u << LOG_STRIDE) - 1u);
    base = ((q >> LOG_STRIDE) << (LOG_L - S0)) + o;
  }
};

// One shared-memory round, in place.
template <class F, int LOG_L, int S0, int R>
__device__ __forceinline__ void round_smem(uint32_t* buf, const uint32_t* tw) {
  using G = RoundGeo<LOG_L, S0, R>;
#pragma unroll
  for (int j = 0; j < G::PER_THREAD; j++) {
    uint32_t line, o, base;
    G::item(threadIdx.x + j * kThreads, line, o, base);
    uint32_t v[1 << R];
    constexpr uint32_t ST = sstep<G::LOG_LW, G::LOG_STRIDE>();
    uint32_t* row = buf + set_row<G::LOG_LW, G::LOG_STRIDE, (1 << R)>(base, line);
#pragma unroll
    for (int k = 0; k < (1 << R); k++) v[k] = row[k * ST];
    dif<F, LOG_L, S0, R>(v, o, tw);
#pragma unroll
    for (int k = 0; k < (1 << R); k++) row[k * ST] = v[k];
  }
}

// Round plan.  Inverse: a first round of four, one short round (l mod 4
// stages), rounds of four, and a last round of four at stride 1 that stays
// in registers (for l < 8: the short round, then the last).  Forward: the
// fused first round of four, rounds of four, one short round, then a last
// round of four at stride 1 (for l < 8 the short round is the last).  Only
// first rounds touch stages 0..3.
template <int LOG_L, int S0>
constexpr int inv_round_r() {
  if constexpr (LOG_L < 8) return S0 == 0 ? LOG_L - 4 : 4;
  return (S0 == 4 && LOG_L % 4) ? LOG_L % 4 : 4;
}
template <int LOG_L>
constexpr int fwd_last_r() {
  return LOG_L <= 4 ? LOG_L : (LOG_L < 8 ? LOG_L - 4 : 4);
}

template <class F, int LOG_L, int S0>
__device__ __forceinline__ void inv_middle(uint32_t* buf, const uint32_t* tw) {
  if constexpr (S0 + 4 < LOG_L) {
    constexpr int R = inv_round_r<LOG_L, S0>();
    round_smem<F, LOG_L, S0, R>(buf, tw);
    __syncthreads();
    inv_middle<F, LOG_L, S0 + R>(buf, tw);
  }
}
template <class F, int LOG_L, int S0>
__device__ __forceinline__ void fwd_middle(uint32_t* buf, const uint32_t* tw) {
  constexpr int SLAST = LOG_L - fwd_last_r<LOG_L>();
  if constexpr (S0 < SLAST) {
    constexpr int R = SLAST - S0 < 4 ? SLAST - S0 : 4;
    round_smem<F, LOG_L, S0, R>(buf, tw);
    __syncthreads();
    fwd_middle<F, LOG_L, S0 + R>(buf, tw);
  }
}

// Forward last round (stride 1): sets of 2^RLAST consecutive positions go to
// store(line, first position, values).
template <class F, int LOG_L, class Store>
__device__ __forceinline__ void fwd_last(const uint32_t* buf, const uint32_t* tw, Store store) {
  constexpr int RL = fwd_last_r<LOG_L>();
  constexpr int SL = LOG_L - RL;
  using G = RoundGeo<LOG_L, SL, RL>;
#pragma unroll
  for (int j = 0; j < G::PER_THREAD; j++) {
    uint32_t line, o, base;
    G::item(threadIdx.x + j * kThreads, line, o, base);
    uint32_t v[1 << RL];
    constexpr uint32_t ST = sstep<G::LOG_LW, 0>();
    const uint32_t* row = buf + set_row<G::LOG_LW, 0, (1 << RL)>(base, line);
#pragma unroll
    for (int k = 0; k < (1 << RL); k++) v[k] = row[k * ST];
    dif<F, LOG_L, SL, RL>(v, 0u, tw);
    store(line, base, v);
  }
}

struct TileCtx {
  uint32_t log_ws, col0, g0, n_other, w;
};
__device__ __forceinline__ TileCtx tile_ctx(const PassGeom& g, uint32_t local, uint32_t w) {
  TileCtx t;
  t.log_ws = g.log_ws;
  t.col0 = (local % g.n_ct) << g.log_ws;
  t.g0 = ((local / g.n_ct) % g.groups) << g.log_J;
  t.n_other = 1u << g.log_other;
  t.w = w;
  return t;
}
// Column and sub-transform of a line; inactive lines are past the matrix.
__device__ __forceinline__ bool line_at(const TileCtx& T, uint32_t line, uint32_t& col, uint32_t& sub) {
  col = T.col0 + (line & ((1u << T.log_ws) - 1u));
  sub = T.g0 + (line >> T.log_ws);
  return col < T.w && sub < T.n_other;
}

struct NoTwist {
  static constexpr bool active = false;
  __device__ __forceinline__ uint2 operator()(uint32_t, uint32_t, uint32_t) const { return make_uint2(0, 0); }
};

// Four-step twiddle w_n^(+-s x) on a first round's loads, s the line's
// sub-transform and x = o + k * stride the position: {w^(s o), w^(s stride)}.
template <class F, bool INV>
struct LineTwist {
  const TwiddleTables* tw;
  const TileCtx* T;
  uint32_t log_n, n_mask;
  static constexpr bool active = true;
  __device__ __forceinline__ uint2 operator()(uint32_t o, uint32_t line, uint32_t log_stride) const {
    const uint32_t sub = T->g0 + (line >> T->log_ws);
    return make_uint2(omega<F>(*tw, log_n, (sub * o) & n_mask, INV),
                      omega<F>(*tw, log_n, (sub << log_stride) & n_mask, INV));
  }
};

// Loads the 2^R elements of a first-round set from global memory: line
// base `p` (nullptr: inactive line, zeros), element k at p + (o + k * stride)
// * pos_step, times a * q^k when `twist` is active.
template <class F, int R, int LOG_STRIDE, class Twist>
__device__ __forceinline__ void load_set(uint32_t* v, const uint32_t* p, uint32_t o, uint32_t line,
                                         uint64_t pos_step, const Twist& twist) {
  if (p) {
    p += (uint64_t)o * pos_step;
    const uint64_t step = pos_step << LOG_STRIDE;
    if (set_in_range<(1 << R)>(p, step, s_in, kGuardLoad)) {
#pragma unroll
      for (int k = 0; k < (1 << R); k++) v[k] = __ldg(p + k * step);
    } else {
#pragma unroll
      for (int k = 0; k < (1 << R); k++) v[k] = 0u;
    }
    if constexpr (Twist::active) {
      const uint2 aq = twist(o, line, (uint32_t)LOG_STRIDE);
      uint32_t cur = aq.x;
#pragma unroll
      for (int k = 0; k < (1 << R); k++) {
        v[k] = Fp<F>::mul(v[k], cur);
        if (k + 1 < (1 << R)) cur = Fp<F>::mul(cur, aq.y);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < (1 << R); k++) v[k] = 0u;
  }
}

// First round (stages 0 .. R-1) from global memory into shared memory.
template <class F, int LOG_L, int R, class LineBase, class Twist>
__device__ __forceinline__ void first_round_global(uint32_t* buf, const uint32_t* tw, LineBase line_base,
                                                   uint64_t pos_step, const Twist& twist) {
  using G = RoundGeo<LOG_L, 0, R>;
#pragma unroll
  for (int j = 0; j < G::PER_THREAD; j++) {
    uint32_t line, o, base;
    G::item(threadIdx.x + j * kThreads, line, o, base);
    uint32_t v[1 << R];
    load_set<F, R, G::LOG_STRIDE>(v, line_base(line), o, line, pos_step, twist);
    dif<F, LOG_L, 0, R>(v, o, tw);
    constexpr uint32_t ST = sstep<G::LOG_LW, G::LOG_STRIDE>();
    uint32_t* row = buf + set_row<G::LOG_LW, G::LOG_STRIDE, (1 << R)>(base, line);
#pragma unroll
    for (int k = 0; k < (1 << R); k++) row[k * ST] = v[k];
  }
}

// Inverse transform of the whole tile with its last round (2^RL consecutive
// positions, RL = min(l, 4)) left in registers: thread t's coef[k] is
// position 2^RL q + k of line `line` (one set per thread).
template <class F, int LOG_L, class LineBase, class Twist>
__device__ __forceinline__ void inverse_to_regs(uint32_t* buf, const uint32_t* twi, LineBase line_base,
                                                uint64_t pos_step, const Twist& twist, uint32_t* coef,
                                                uint32_t& line, uint32_t& q) {
  constexpr int RL = LOG_L < 4 ? LOG_L : 4;
  constexpr int SL = LOG_L - RL;
  using G = RoundGeo<LOG_L, SL, RL>;
  static_assert(G::N_ITEMS == kThreads, "one last-round set per thread");
  uint32_t o, base;
  G::item(threadIdx.x, line, o, base);
  q = base >> RL;
  if constexpr (SL > 0) {
    constexpr int R0 = inv_round_r<LOG_L, 0>();
    first_round_global<F, LOG_L, R0>(buf, twi, line_base, pos_step, twist);
    __syncthreads();
    inv_middle<F, LOG_L, R0>(buf, twi);
    constexpr uint32_t ST = sstep<G::LOG_LW, 0>();
    const uint32_t* row = buf + set_row<G::LOG_LW, 0, (1 << RL)>(base, line);
#pragma unroll
    for (int k = 0; k < (1 << RL); k++) coef[k] = row[k * ST];
  } else {
    load_set<F, RL, 0>(coef, line_base(line), 0u, line, pos_step, twist);
  }
  dif<F, LOG_L, SL, RL>(coef, 0u, twi);
}

// Forward transform whose first round takes the inverse's last-round
// registers: the input at natural position o + k * stride (o = rev(q)) is
// coef[rev(k)] * a * q^k, {a, q} = scale(o, line).  Later rounds run in
// shared memory; the last hands its sets to `store`.
template <class F, int LOG_L, class Scale, class Store>
__device__ __forceinline__ void forward_from_regs(uint32_t* buf, const uint32_t* twf, const uint32_t* coef,
                                                  uint32_t line, uint32_t q, Scale scale, Store store) {
  constexpr int RF = LOG_L < 4 ? LOG_L : 4;
  constexpr int LOG_STRIDE = LOG_L - RF;
  using G = RoundGeo<LOG_L, 0, RF>;
  const uint32_t o = LOG_STRIDE ? (__brev(q) >> (32 - LOG_STRIDE)) : 0u;
  uint32_t v[1 << RF];
  const uint2 aq = scale(o, line);
  uint32_t cur = aq.x;
#pragma unroll
  for (int k = 0; k < (1 << RF); k++) {
    v[k] = Fp<F>::mul(coef[rev_bits(k, RF)], cur);
    if (k + 1 < (1 << RF)) cur = Fp<F>::mul(cur, aq.y);
  }
  dif<F, LOG_L, 0, RF>(v, o, twf);
  if constexpr (RF == LOG_L) {
    store(line, 0u, v);
  } else {
    __syncthreads();  // shared memory may still be read by the previous phase
    constexpr uint32_t ST = sstep<G::LOG_LW, LOG_STRIDE>();
    uint32_t* row = buf + set_row<G::LOG_LW, LOG_STRIDE, (1 << RF)>(o, line);
#pragma unroll
    for (int k = 0; k < (1 << RF); k++) row[k * ST] = v[k];
    __syncthreads();
    fwd_middle<F, LOG_L, RF>(buf, twf);
    fwd_last<F, LOG_L>(buf, twf, store);
  }
}

// ---------------------------------------------------------------------------
// One-pass form: tile = all n rows of up to LW columns.
template <class F, int LOG_L>
__global__ void __launch_bounds__(kThreads, 1) k_lde_small(const __grid_constant__ LdeBatch batch,
                                                           const __grid_constant__ TwiddleTables tw) {
  constexpr int LOG_LW = (int)tile_log_lw(LOG_L);
  constexpr uint32_t L = 1u << LOG_L;
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassSmall, blockIdx.x, local);
  s_in = GuardRange{M.in, M.in + (((uint64_t)M.w << M.log_n))};
  s_out = GuardRange{M.out, M.out + (((uint64_t)M.w << (M.log_n + lde_log_c(M))))};
  s_smem_words = tile_words_l(LOG_L);
  const TileCtx T = tile_ctx(pass_geom(M, kPassSmall), local, M.w);
  const uint32_t w = M.w;
  if constexpr (LOG_L == 0) {
    // height 1: every LDE row equals the input row (the scale g^0 / 1 is 1)
    uint32_t col, sub;
    if (line_at(T, threadIdx.x, col, sub))
      for (uint32_t cb = 0; cb < (1u << lde_log_c(M)); cb++) {
        const uint32_t* pi = M.in + col;
        uint32_t* po = M.out + (uint64_t)cb * w + col;
        if (pi < M.in || pi >= M.in + w) { guard_trip(kGuardLoad, col, w); continue; }
        if (po < M.out || po >= M.out + ((uint64_t)w << lde_log_c(M))) { guard_trip(kGuardStore, (uint64_t)cb * w + col, (uint64_t)w << lde_log_c(M)); continue; }
        *po = __ldg(pi);
      }
  } else {
    uint32_t* buf = smem;
    uint32_t* twf = buf + tile_words_l(LOG_L);
    uint32_t* twi = twf + 2 * L;
    load_twiddles<LOG_L>(twf, tw, false);
    load_twiddles<LOG_L>(twi, tw, true);
    __syncthreads();
    auto line_base = [&](uint32_t line) -> const uint32_t* {
      uint32_t col, sub;
      return line_at(T, line, col, sub) ? M.in + col : nullptr;
    };
    uint32_t coef[16], line, q;
    inverse_to_regs<F, LOG_L>(buf, twi, line_base, (uint64_t)w, NoTwist(), coef, line, q);
    constexpr int RF = LOG_L < 4 ? LOG_L : 4;
    constexpr int RL = fwd_last_r<LOG_L>();
    const uint32_t nm = n_monty<F>(LOG_L);
    for (uint32_t cb = 0; cb < (1u << lde_log_c(M)); cb++) {
      const uint32_t* pt = pw_table(M, cb);
      // coefficient i scales by g^i / n: {g^o / n, g^stride} along a set
      // (table entries carry the 1/n, so the step is multiplied back by n)
      const uint32_t step = Fp<F>::mul(pw_at<F>(pt, 1u << (LOG_L - RF)), nm);
      uint32_t* outb = M.out + (uint64_t)cb * L * w;
      forward_from_regs<F, LOG_L>(
          buf, twf, coef, line, q, [&](uint32_t o, uint32_t) { return make_uint2(pw_at<F>(pt, o), step); },
          [&](uint32_t ln, uint32_t base, const uint32_t* v) {
            uint32_t col, sub;
            if (!line_at(T, ln, col, sub)) return;
            uint32_t* p = outb + (uint64_t)base * w + col;
            if (set_in_range<(1 << RL)>(p, w, s_out, kGuardStore)) {
#pragma unroll
              for (int k = 0; k < (1 << RL); k++) p[(uint64_t)k * w] = v[k];
            }
          });
    }
  }
}

// Pass A: rows j2 + n2 * j1 of the input -> T1 rows k1 * n2 + j2.
template <class F, int LOG_L>
__global__ void __launch_bounds__(kThreads, 2) k_lde_a(const __grid_constant__ LdeBatch batch,
                                                       const __grid_constant__ TwiddleTables tw) {
  constexpr int LOG_LW = (int)tile_log_lw(LOG_L);
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassA, blockIdx.x, local);
  s_in = GuardRange{M.in, M.in + (((uint64_t)M.w << M.log_n))};
  s_out = GuardRange{M.t1, M.t1 + (((uint64_t)M.w << M.log_n))};
  s_smem_words = tile_words_l(LOG_L);
  const TileCtx T = tile_ctx(pass_geom(M, kPassA), local, M.w);
  const uint32_t w = M.w, log_n2 = M.log_n2;
  uint32_t* buf = smem;
  uint32_t* twi = buf + tile_words_l(LOG_L);
  load_twiddles<LOG_L>(twi, tw, true);
  __syncthreads();
  auto line_base = [&](uint32_t line) -> const uint32_t* {
    uint32_t col, sub;
    return line_at(T, line, col, sub) ? M.in + (uint64_t)sub * w + col : nullptr;
  };
  uint32_t coef[16], line, q;
  inverse_to_regs<F, LOG_L>(buf, twi, line_base, (uint64_t)w << log_n2, NoTwist(), coef, line, q);
  // positions 16 q + k hold frequencies k1 = rev(q) + rev4(k) * 2^(l-4)
  uint32_t col, j2;
  if (line_at(T, line, col, j2)) {
    const uint32_t k1_0 = __brev(q) >> (32 - (LOG_L - 4));
    uint32_t* p = M.t1 + ((((uint64_t)k1_0 << log_n2) + j2) * w + col);
    const uint64_t step = ((uint64_t)w << log_n2) << (LOG_L - 4);
    if (set_in_range<16>(p, step, s_out, kGuardStore)) {
#pragma unroll
      for (int kr = 0; kr < 16; kr++) p[kr * step] = coef[rev_bits(kr, 4)];
    }
  }
}

// Pass B: T1 rows k1 * n2 + j2 times w_n^-(j2 k1) -> coefficients -> per
// coset -> T2 (the twiddle w_n^(k1 k1') is applied by pass C on its loads).
template <class F, int LOG_L>
__global__ void __launch_bounds__(kThreads, 2) k_lde_b(const __grid_constant__ LdeBatch batch,
                                                       const __grid_constant__ TwiddleTables tw) {
  constexpr int LOG_LW = (int)tile_log_lw(LOG_L);
  constexpr uint32_t L = 1u << LOG_L;
  constexpr int RL = fwd_last_r<LOG_L>();
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassB, blockIdx.x, local);
  s_in = GuardRange{M.t1, M.t1 + (((uint64_t)M.w << M.log_n))};
  s_out = GuardRange{M.t2, M.t2 + (((uint64_t)M.w << (M.log_n + lde_log_c(M))))};
  s_smem_words = tile_words_l(LOG_L);
  const TileCtx T = tile_ctx(pass_geom(M, kPassB), local, M.w);
  const uint32_t w = M.w, log_n1 = M.log_n1;
  const uint64_t n = 1ull << M.log_n;
  uint32_t* buf = smem;
  uint32_t* twf = buf + tile_words_l(LOG_L);
  uint32_t* twi = twf + 2 * L;
  load_twiddles<LOG_L>(twf, tw, false);
  load_twiddles<LOG_L>(twi, tw, true);
  __syncthreads();
  auto line_base = [&](uint32_t line) -> const uint32_t* {
    uint32_t col, sub;
    return line_at(T, line, col, sub) ? M.t1 + ((uint64_t)sub << LOG_L) * w + col : nullptr;
  };
  const LineTwist<F, true> twist{&tw, &T, M.log_n, (uint32_t)(n - 1)};
  uint32_t coef[16], line, q;
  inverse_to_regs<F, LOG_L>(buf, twi, line_base, (uint64_t)w, twist, coef, line, q);
  const uint32_t nm = n_monty<F>(M.log_n);
  for (uint32_t cb = 0; cb < (1u << lde_log_c(M)); cb++) {
    const uint32_t* pt = pw_table(M, cb);
    // coefficient i = k1 + n1 * p scales by g^i / n: {g^(k1 + n1 o) / n, g^(n1 stride)}
    const uint32_t step = Fp<F>::mul(pw_at<F>(pt, 1u << (LOG_L - 4 + log_n1)), nm);
    uint32_t* t2 = M.t2 + (uint64_t)cb * n * w;
    forward_from_regs<F, LOG_L>(
        buf, twf, coef, line, q,
        [&](uint32_t o, uint32_t ln) {
          return make_uint2(pw_at<F>(pt, T.g0 + (ln >> T.log_ws) + (o << log_n1)), step);
        },
        [&](uint32_t ln, uint32_t base, const uint32_t* v) {
          uint32_t col, k1;
          if (!line_at(T, ln, col, k1)) return;
          // positions base + k hold k1' = rev(base) + rev_RL(k) * 2^(l - RL)
          const uint32_t k1p_0 = __brev(base) >> (32 - LOG_L);
          uint32_t* p = t2 + ((((uint64_t)k1p_0 << log_n1) + k1) * w + col);
          const uint64_t step2 = ((uint64_t)w << log_n1) << (LOG_L - RL);
          if (set_in_range<(1 << RL)>(p, step2, s_out, kGuardStore)) {
#pragma unroll
            for (int kr = 0; kr < (1 << RL); kr++) p[kr * step2] = v[rev_bits(kr, RL)];
          }
        });
  }
}

// Pass C: T2 rows cb*n + k1' * n1 + k1 times w_n^(k1 k1') -> out rows
// cb*n + rev(k1') * n1 + j.
template <class F, int LOG_L>
__global__ void __launch_bounds__(kThreads, 2) k_lde_c(const __grid_constant__ LdeBatch batch,
                                                       const __grid_constant__ TwiddleTables tw) {
  constexpr int LOG_LW = (int)tile_log_lw(LOG_L);
  constexpr int RL = fwd_last_r<LOG_L>();
  static_assert(LOG_L > 4, "three-pass sub-transforms have at least 2^6 points");
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassC, blockIdx.x, local);
  s_in = GuardRange{M.t2, M.t2 + (((uint64_t)M.w << (M.log_n + lde_log_c(M))))};
  s_out = GuardRange{M.out, M.out + (((uint64_t)M.w << (M.log_n + lde_log_c(M))))};
  s_smem_words = tile_words_l(LOG_L);
  const PassGeom g = pass_geom(M, kPassC);
  const TileCtx T = tile_ctx(g, local, M.w);
  const uint32_t w = M.w, log_n2 = M.log_n2;
  const uint32_t cb = local / (g.n_ct * g.groups);
  const uint64_t n = 1ull << M.log_n;
  uint32_t* buf = smem;
  uint32_t* twf = buf + tile_words_l(LOG_L);
  load_twiddles<LOG_L>(twf, tw, false);
  __syncthreads();
  const uint32_t* src = M.t2 + (uint64_t)cb * n * w;
  uint32_t* dst = M.out + (uint64_t)cb * n * w;
  auto line_base = [&](uint32_t line) -> const uint32_t* {
    uint32_t col, sub;
    return line_at(T, line, col, sub) ? src + ((uint64_t)sub << LOG_L) * w + col : nullptr;
  };
  const LineTwist<F, false> twist{&tw, &T, M.log_n, (uint32_t)(n - 1)};
  first_round_global<F, LOG_L, 4>(buf, twf, line_base, (uint64_t)w, twist);
  __syncthreads();
  fwd_middle<F, LOG_L, 4>(buf, twf);
  fwd_last<F, LOG_L>(buf, twf, [&](uint32_t ln, uint32_t base, const uint32_t* v) {
    uint32_t col, k1p;
    if (!line_at(T, ln, col, k1p)) return;
    const uint64_t row = ((uint64_t)(__brev(k1p) >> (32 - log_n2)) << LOG_L) + base;
    uint32_t* p = dst + row * w + col;
    if (set_in_range<(1 << RL)>(p, w, s_out, kGuardStore)) {
#pragma unroll
      for (int k = 0; k < (1 << RL); k++) p[(uint64_t)k * w] = v[k];
    }
  });
}

// ---------------------------------------------------------------------------
// Power tables of matrix blockIdx.y: for the cb-th coset block it computes
// (global block cb0 + cb), entries [0, 4096) hold g^e / n and [4096, 8192)
// hold g^(4096 e), g = shift * w_N^rev_b(cb0 + cb).
template <class F>
__global__ void k_pow_tables(const __grid_constant__ LdeBatch batch, const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  const LdeMat& M = batch.m[blockIdx.y];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (kPwWords << lde_log_c(M))) return;
  const uint32_t cb = i / kPwWords, e = i % kPwWords;
  const uint32_t log_N = M.log_n + M.log_b;
  const uint32_t g = B::mul(M.shift, omega<F>(tw, log_N, bitrev32(lde_cb0(M) + cb, M.log_b), false));
  uint32_t v;
  if (e < 4096u) {
    // 1/2^log_n = p - (p - 1) / 2^log_n (canonical), since 2^log_n * ((p-1)/2^log_n) = -1
    const uint32_t ninv = B::to_monty(F::P - ((F::P - 1u) >> M.log_n));
    v = B::mul(B::pow(g, e), ninv);
  } else {
    v = B::pow(g, (uint64_t)(e - 4096u) << 12);
  }
  if (i >= (kPwWords << lde_log_c(M))) { guard_trip(kGuardStore, i, kPwWords << lde_log_c(M)); return; }
  M.pw[i] = v;
}

bool lde_split_valid(uint32_t log_n, uint32_t log_n1) {
  return log_n > (uint32_t)kLdeSmallMaxLog && log_n <= kLdeMaxLogN && log_n1 >= (uint32_t)kMinLogL3 &&
         log_n1 <= (uint32_t)kMaxLogL && log_n - log_n1 >= (uint32_t)kMinLogL3 && log_n - log_n1 <= (uint32_t)kMaxLogL;
}

void plan_lde_tiling(LdeMat& m, uint32_t log_n1) {
  if ((int)m.log_n <= kLdeSmallMaxLog) {
    m.log_n1 = m.log_n2 = 0;
  } else if (lde_split_valid(m.log_n, log_n1)) {
    m.log_n1 = log_n1;
    m.log_n2 = m.log_n - log_n1;
  } else {
    m.log_n1 = (m.log_n + 1) / 2;
    m.log_n2 = m.log_n / 2;
  }
}

// Dynamic shared memory of a pass at sub-transform length 2^log_L (bytes):
// the tile plus one (passes A, C) or two (one-pass, B) twiddle tables of L
// two-word entries (L - 1 used).  At most 8704 + 4 * 4096 words (98 KiB), so
// two CTAs fit an SM.
static size_t smem_bytes(uint32_t log_L, int pass) {
  const size_t L = 1ull << log_L;
  const size_t tile = tile_words_l(log_L);
  const size_t tw_words = (pass == kPassA || pass == kPassC) ? 2 * L : 4 * L;
  return (tile + tw_words) * 4;
}
constexpr int kSmemCap = 100 * 1024;
static_assert((tile_words_l(12) + 4 * (1u << 12)) * 4 <= (uint32_t)kSmemCap, "largest pass fits the cap");

// ---- dispatch over the template parameter LOG_L ----------------------------
template <class F, int LOG_L>
static cudaError_t set_attrs_from() {
  const int cap = kSmemCap;
  cudaError_t e = cudaSuccess;
  if constexpr (LOG_L <= kLdeSmallMaxLog) {
    if ((e = cudaFuncSetAttribute(k_lde_small<F, LOG_L>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  }
  if constexpr (LOG_L >= kMinLogL3) {
    if ((e = cudaFuncSetAttribute(k_lde_a<F, LOG_L>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
    if ((e = cudaFuncSetAttribute(k_lde_b<F, LOG_L>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
    if ((e = cudaFuncSetAttribute(k_lde_c<F, LOG_L>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap))) return e;
  }
  if constexpr (LOG_L < kMaxLogL) e = set_attrs_from<F, LOG_L + 1>();
  return e;
}

template <class F>
static cudaError_t set_smem_attrs() {
  static std::atomic<uint64_t> done_mask{0};  // one bit per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return cudaSuccess;
  if ((e = set_attrs_from<F, 0>())) return e;
  done_mask.fetch_or(bit);
  return cudaSuccess;
}

template <class F, int LOG_L = 0>
static void launch_pass(uint32_t log_L, int pass, uint32_t grid, size_t smem, const LdeBatch& b,
                        const TwiddleTables& tw, cudaStream_t st) {
  if (log_L == (uint32_t)LOG_L) {
    if (pass == kPassSmall) {
      if constexpr (LOG_L <= kLdeSmallMaxLog) k_lde_small<F, LOG_L><<<grid, kThreads, smem, st>>>(b, tw);
    } else if constexpr (LOG_L >= kMinLogL3) {
      if (pass == kPassA) k_lde_a<F, LOG_L><<<grid, kThreads, smem, st>>>(b, tw);
      if (pass == kPassB) k_lde_b<F, LOG_L><<<grid, kThreads, smem, st>>>(b, tw);
      if (pass == kPassC) k_lde_c<F, LOG_L><<<grid, kThreads, smem, st>>>(b, tw);
    }
    return;
  }
  if constexpr (LOG_L < kMaxLogL) launch_pass<F, LOG_L + 1>(log_L, pass, grid, smem, b, tw, st);
}

template <class F>
static cudaError_t launch_lde_t(const LdeMat* mats, uint32_t n_mats, TwiddleTables tw, cudaStream_t st,
                                uint64_t* launches) {
  cudaError_t e = set_smem_attrs<F>();
  if (e) return e;
  for (uint32_t k = 0; k < n_mats; k++) {
    const LdeMat& m = mats[k];
    const bool one_pass = m.log_n1 == 0;
    if ((one_pass && m.log_n > (uint32_t)kLdeSmallMaxLog) ||
        (!one_pass && (m.log_n > kLdeMaxLogN || m.log_n1 > (uint32_t)kMaxLogL ||
                       m.log_n2 < (uint32_t)kMinLogL3 || m.log_n1 + m.log_n2 != m.log_n)))
      return cudaErrorInvalidValue;
  }
  for (uint32_t base = 0; base < n_mats; base += kLdeBatch) {
    LdeBatch all;
    memset(&all, 0, sizeof all);
    all.n = std::min<uint32_t>(kLdeBatch, n_mats - base);
    uint32_t max_b = 0;
    for (uint32_t k = 0; k < all.n; k++) {
      all.m[k] = mats[base + k];
      max_b = std::max(max_b, lde_log_c(all.m[k]));
    }
    dim3 pgrid((kPwWords << max_b) / 256, all.n);
    k_pow_tables<F><<<pgrid, 256, 0, st>>>(all, tw);
    if ((e = cudaGetLastError())) return e;
    if (launches) *launches += 1;
    // passes in order; within a pass one launch per sub-transform length
    for (int pass = kPassSmall; pass <= kPassC; pass++) {
      for (uint32_t lL = 0; lL <= (uint32_t)kMaxLogL; lL++) {
        LdeBatch sub;
        memset(&sub, 0, sizeof sub);
        uint32_t tiles = 0;
        for (uint32_t k = 0; k < all.n; k++) {
          const uint32_t t = lde_tiles(all.m[k], pass);
          if (t && pass_log_L(all.m[k], pass) == lL) {
            sub.m[sub.n++] = all.m[k];
            tiles += t;
          }
        }
        if (!tiles) continue;
        launch_pass<F>(lL, pass, tiles, smem_bytes(lL, pass), sub, tw, st);
        if ((e = cudaGetLastError())) return e;
        if (launches) *launches += 1;
      }
    }
  }
  return cudaSuccess;
}

cudaError_t launch_stage_tables(int field, TwiddleTables tw, uint32_t* stage, cudaStream_t st) {
  const uint32_t n = stage_base(kMaxLogL + 1);
  if (field == 0)
    k_stage_tables<KoalaBear><<<(n + 255) / 256, 256, 0, st>>>(tw, stage);
  else
    k_stage_tables<BabyBear><<<(n + 255) / 256, 256, 0, st>>>(tw, stage);
  return cudaGetLastError();
}

cudaError_t lde_guard_fetch(GuardRecord* dst, cudaStream_t st) {
  return cudaMemcpyFromSymbolAsync(dst, g_lde_guard, sizeof(GuardRecord), 0, cudaMemcpyDeviceToHost, st);
}
cudaError_t lde_guard_clear() {
  const GuardRecord z{};
  return cudaMemcpyToSymbol(g_lde_guard, &z, sizeof z);
}

cudaError_t launch_lde(int field, const LdeMat* mats, uint32_t n_mats, TwiddleTables tw, cudaStream_t st,
                       uint64_t* launches) {
  if (field == 0) return launch_lde_t<KoalaBear>(mats, n_mats, tw, st, launches);
  return launch_lde_t<BabyBear>(mats, n_mats, tw, st, launches);
}

}  // namespace pico
