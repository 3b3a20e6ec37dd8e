// Batched coset low-degree extension (Radix2DitParallel::coset_lde_batch
// followed by the row bit-reversal of TwoAdicFriPcs::commit).
//
// Per matrix: evaluations e on H_n (n x w, row-major) -> coefficients
// c = iNTT(e) -> d_i = c_i * g_cb^i for each coset block cb in [0, 2^b) with
// g_cb = shift * w_N^rev_b(cb) -> NTT_n(d) in bit-reversed order.  Output row
// cb*n + j then holds f(shift * w_N^rev_N(cb*n + j)), i.e. committed row i is
// f(shift * w_N^rev(i)) (vm/src/compiler/recursion/circuit/fri.rs:155-171).
//
// Tiles.  A CTA stages a tile of L = 2^l positions x LW lines in shared memory
// (L * LW <= 2^13 words, 32 KiB); a line is one column of one sub-transform
// (J adjacent sub-transforms x ws adjacent columns).  Sub-transforms are
// decimation-in-frequency (natural in, bit-reversed out) and run in rounds of
// up to four radix-2 stages held in registers: a thread loads the 2^r
// elements a round combines, applies r stages, and stores them back, so
// shared memory sees one round trip per four stages.  Shared addresses are
// XOR-swizzled so the stride-1 rounds do not conflict on banks.
//
// Fusion.  The inverse transform's last round works on 16 consecutive
// positions; those 16 values are exactly the 16 inputs of the forward
// transform's first round (in bit-reversed order), so the coefficients stay
// in registers between the two transforms and are reused for every coset.
//
// One-pass form (n <= 2^11): global -> inverse -> per coset: scale, forward
// -> global.  Three-pass form, n = n1 * n2 (four-step):
//   A: iNTT_n1 over j1 for each j2, twiddle w_n^-(j2 k1)           -> T1[k1*n2 + j2]
//   B: iNTT_n2 over j2 -> coefficients c[k1 + n1 k2]; per coset: scale,
//      NTT_n2 over k2, twiddle w_n^(k1 k1')                         -> T2[cb*n + k1'*n1 + k1]
//   C: NTT_n1 over k1 -> bit-reversed block                         -> out[cb*n + rev(k1')*n1 + j]
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "field.cuh"
#include "internal.h"

namespace pico {

constexpr uint32_t kLogTile = 13;  // words per tile: 2^13 (32 KiB)
constexpr uint32_t kThreads = 512;
constexpr uint32_t kMaxSetsPerThread = 1;  // (2^13 / 16) / 512

constexpr int rev_bits(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

enum LdePass { kPassSmall = 0, kPassA = 1, kPassB = 2, kPassC = 3 };

PICO_HD uint32_t ceil_log2(uint32_t x) {
  uint32_t l = 0;
  while ((1u << l) < x) l++;
  return l;
}

// Tile shape of a pass: sub-transform length 2^log_L, `log_other`
// sub-transforms available side by side; returns log2 of columns per tile
// (ws) and of adjacent sub-transforms per tile (J).
PICO_HD void tile_shape(uint32_t log_L, uint32_t w, uint32_t log_other, uint32_t& log_ws, uint32_t& log_J) {
  const uint32_t log_LW = log_L >= kLogTile ? 0u : kLogTile - log_L;
  uint32_t cw = ceil_log2(w > 0 ? w : 1u);
  log_ws = cw < log_LW ? cw : log_LW;
  if (log_ws > 6) log_ws = 6;  // at most 64 columns (256 bytes of a row) per tile
  const uint32_t rest = log_LW - log_ws;
  log_J = rest < log_other ? rest : log_other;
}

struct PassGeom {
  uint32_t log_L, log_other, log_ws, log_J, n_ct, groups;
};

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
  tile_shape(g.log_L, m.w, g.log_other, g.log_ws, g.log_J);
  g.n_ct = (m.w + (1u << g.log_ws) - 1) >> g.log_ws;
  g.groups = 1u << (g.log_other - g.log_J);
  return g;
}

// Tiles of one matrix in one pass (host and device).
PICO_HD uint32_t lde_tiles(const LdeMat& m, int pass) {
  if ((pass == kPassSmall) != (m.log_n1 == 0)) return 0u;
  const PassGeom g = pass_geom(m, pass);
  const uint32_t t = g.groups * g.n_ct;
  return pass == kPassC ? t << m.log_b : t;
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

template <class F>
__device__ void fill_twiddles(uint32_t* t, uint32_t log_L, bool inv, const TwiddleTables& tw) {
  const uint32_t h = (1u << log_L) >> 1;
  for (uint32_t i = threadIdx.x; i < h; i += blockDim.x) t[i] = omega<F>(tw, log_L, i, inv);
}

// Swizzled shared-memory index of (position, line).
__device__ __forceinline__ uint32_t sidx(uint32_t pos, uint32_t line, uint32_t log_LW) {
  const uint32_t mask = ((1u << log_LW) - 1u) & 7u;
  return (pos << log_LW) + (line ^ ((pos >> 4) & mask));
}

// DIF butterfly: (a, b) -> (a + b, (a - b) * w), canonical in and out.
// a - b + p lies in (0, 2p), so the Montgomery product stays below 2p.
template <class F>
__device__ __forceinline__ void bfly(uint32_t& a, uint32_t& b, uint32_t w) {
  using B = Fp<F>;
  const uint32_t x = B::add(a, b);
  const uint32_t d = a - b + F::P;
  b = B::canon(B::redc((uint64_t)d * w));
  a = x;
}

// r = LOGR stages s0 .. s0+r-1 of an L-point DIF on the 2^r elements
// v[k] = x[base + k * stride], stride = L >> (s0 + r), base = blk * (L >> s0) + o.
// tw[t] = w_L^(+-t), t < L/2.
template <class F, int LOGR>
__device__ __forceinline__ void dif_round(uint32_t* v, uint32_t s0, uint32_t o, uint32_t log_L, const uint32_t* tw) {
  constexpr int R = 1 << LOGR;
#pragma unroll
  for (int t = 0; t < LOGR; t++) {
    const int half = R >> (t + 1);
    const uint32_t s = s0 + t;
    const uint32_t obase = o << s;
    const uint32_t kstep = (1u << log_L) >> (LOGR - t);
#pragma unroll
    for (int k = 0; k < R; k++) {
      if (k & half) continue;
      const uint32_t w = tw[obase + (uint32_t)(k & (half - 1)) * kstep];
      bfly<F>(v[k], v[k + half], w);
    }
  }
}

// One shared-memory round: 2^log_L positions x 2^log_LW lines, in place.
template <class F, int LOGR>
__device__ void round_smem(uint32_t* buf, uint32_t s0, uint32_t log_L, uint32_t log_LW, const uint32_t* tw) {
  constexpr int R = 1 << LOGR;
  const uint32_t log_stride = log_L - s0 - LOGR;
  const uint32_t n_items = (1u << (log_L - LOGR)) << log_LW;
  for (uint32_t it = threadIdx.x; it < n_items; it += blockDim.x) {
    const uint32_t line = it & ((1u << log_LW) - 1u);
    const uint32_t q = it >> log_LW;
    const uint32_t o = q & ((1u << log_stride) - 1u);
    const uint32_t base = ((q >> log_stride) << (log_L - s0)) + o;
    uint32_t v[R];
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = buf[sidx(base + ((uint32_t)k << log_stride), line, log_LW)];
    dif_round<F, LOGR>(v, s0, o, log_L, tw);
#pragma unroll
    for (int k = 0; k < R; k++) buf[sidx(base + ((uint32_t)k << log_stride), line, log_LW)] = v[k];
  }
}

template <class F>
__device__ void round_smem_r(int r, uint32_t* buf, uint32_t s0, uint32_t log_L, uint32_t log_LW,
                             const uint32_t* tw) {
  switch (r) {
    case 1: round_smem<F, 1>(buf, s0, log_L, log_LW, tw); break;
    case 2: round_smem<F, 2>(buf, s0, log_L, log_LW, tw); break;
    case 3: round_smem<F, 3>(buf, s0, log_L, log_LW, tw); break;
    default: round_smem<F, 4>(buf, s0, log_L, log_LW, tw); break;
  }
}

// A round whose inputs come from `load(pos, line)` and whose outputs go to
// `store(pos, line, v)`; used for the first and last rounds of a transform.
// For a first round (s0 = 0) `twist(o, line, log_stride)` may return {a, q}: the loaded
// element at position o + k * stride is then multiplied by a * q^k before the
// butterflies (the inter-pass twiddles are geometric along a set).
struct NoTwist {
  __device__ __forceinline__ uint2 operator()(uint32_t, uint32_t, uint32_t) const { return make_uint2(0u, 0u); }
  static constexpr bool active = false;
};

template <class F, int LOGR, class Load, class Store, class Twist>
__device__ __forceinline__ void round_io(uint32_t s0, uint32_t log_L, uint32_t log_LW, const uint32_t* tw,
                                         Load load, Store store, Twist twist) {
  constexpr int R = 1 << LOGR;
  const uint32_t log_stride = log_L - s0 - LOGR;
  const uint32_t n_items = (1u << (log_L - LOGR)) << log_LW;
  for (uint32_t it = threadIdx.x; it < n_items; it += blockDim.x) {
    const uint32_t line = it & ((1u << log_LW) - 1u);
    const uint32_t q = it >> log_LW;
    const uint32_t o = q & ((1u << log_stride) - 1u);
    const uint32_t base = ((q >> log_stride) << (log_L - s0)) + o;
    uint32_t v[R];
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = load(base + ((uint32_t)k << log_stride), line);
    if constexpr (Twist::active) {
      const uint2 aq = twist(o, line, log_stride);
      uint32_t cur = aq.x;
#pragma unroll
      for (int k = 0; k < R; k++) {
        v[k] = Fp<F>::mul(v[k], cur);
        if (k + 1 < R) cur = Fp<F>::mul(cur, aq.y);
      }
    }
    dif_round<F, LOGR>(v, s0, o, log_L, tw);
#pragma unroll
    for (int k = 0; k < R; k++) store(base + ((uint32_t)k << log_stride), line, v[k]);
  }
}

template <class F, class Load, class Store, class Twist = NoTwist>
__device__ __forceinline__ void round_io_r(int r, uint32_t s0, uint32_t log_L, uint32_t log_LW, const uint32_t* tw,
                                           Load load, Store store, Twist twist = Twist()) {
  switch (r) {
    case 1: round_io<F, 1>(s0, log_L, log_LW, tw, load, store, twist); break;
    case 2: round_io<F, 2>(s0, log_L, log_LW, tw, load, store, twist); break;
    case 3: round_io<F, 3>(s0, log_L, log_LW, tw, load, store, twist); break;
    default: round_io<F, 4>(s0, log_L, log_LW, tw, load, store, twist); break;
  }
}

// Round sizes: the inverse puts the short round first (so its last round
// spans 16 consecutive positions); the forward puts it last.
__device__ __forceinline__ int inv_round_size(uint32_t log_L, uint32_t s0) {
  const uint32_t rem = log_L & 3u;
  if (s0 == 0 && rem) return (int)rem;
  const uint32_t left = log_L - s0;
  return left < 4 ? (int)left : 4;
}
__device__ __forceinline__ int fwd_round_size(uint32_t log_L, uint32_t s0) {
  const uint32_t left = log_L - s0;
  return left < 4 ? (int)left : 4;
}

template <class F>
__device__ __forceinline__ void dif_round_r(int r, uint32_t* v, uint32_t s0, uint32_t o, uint32_t log_L,
                                            const uint32_t* tw) {
  switch (r) {
    case 1: dif_round<F, 1>(v, s0, o, log_L, tw); break;
    case 2: dif_round<F, 2>(v, s0, o, log_L, tw); break;
    case 3: dif_round<F, 3>(v, s0, o, log_L, tw); break;
    default: dif_round<F, 4>(v, s0, o, log_L, tw); break;
  }
}

// Inverse DIF over the whole tile: first round from `load`, middle rounds in
// shared memory, last round left in registers coef[j][k] for the thread's
// items j (item = threadIdx.x + j * blockDim.x; each a set of 2^r_last
// consecutive positions).  Requires log_L >= 1.  Returns r_last (4, or log_L
// when log_L < 4).
template <class F, class Load, class Twist = NoTwist>
__device__ int inverse_to_regs(uint32_t* buf, uint32_t log_L, uint32_t log_LW, const uint32_t* twi, Load load,
                               uint32_t coef[kMaxSetsPerThread][16], Twist twist = Twist()) {
  uint32_t s0 = 0;
  const int r_last = log_L < 4 ? (int)log_L : 4;
  const uint32_t s_last = log_L - (uint32_t)r_last;
  if (s_last > 0) {
    const int r0 = inv_round_size(log_L, 0);
    round_io_r<F>(r0, 0, log_L, log_LW, twi, load,
                  [&](uint32_t pos, uint32_t line, uint32_t v) { buf[sidx(pos, line, log_LW)] = v; }, twist);
    s0 = (uint32_t)r0;
    __syncthreads();
    while (s0 < s_last) {
      const int r = inv_round_size(log_L, s0);
      round_smem_r<F>(r, buf, s0, log_L, log_LW, twi);
      s0 += (uint32_t)r;
      __syncthreads();
    }
  }
  const uint32_t n_items = (1u << (log_L - r_last)) << log_LW;
#pragma unroll
  for (uint32_t j = 0; j < kMaxSetsPerThread; j++) {
    const uint32_t it = threadIdx.x + j * blockDim.x;
    if (it < n_items) {
      const uint32_t line = it & ((1u << log_LW) - 1u);
      const uint32_t base = (it >> log_LW) << r_last;
      uint32_t* v = coef[j];
#pragma unroll
      for (int k = 0; k < 16; k++)
        if (k < (1 << r_last)) {
          const uint32_t pos = base + (uint32_t)k;
          v[k] = s0 == 0 ? load(pos, line) : buf[sidx(pos, line, log_LW)];
        }
      if constexpr (Twist::active) {
        if (s0 == 0) {  // single round: this is also the first round (stride 1, o = 0)
          const uint2 aq = twist(0u, line, 0u);
          uint32_t cur = aq.x;
#pragma unroll
          for (int k = 0; k < 16; k++)
            if (k < (1 << r_last)) {
              v[k] = Fp<F>::mul(v[k], cur);
              cur = Fp<F>::mul(cur, aq.y);
            }
        }
      }
      dif_round_r<F>(r_last, v, s0, 0, log_L, twi);
    }
  }
  return r_last;
}

// Forward DIF over the tile whose first-round inputs come from the inverse's
// last-round registers: item j's input at natural position p = o + k*stride
// is coef[j][rev(k)] * a * q^k with {a, q} = scale(o, line) and
// o = rev(item's set index).
// Later rounds run in shared memory; the last round hands (pos, line,
// value) to `store`.  RF (the first round's size) is a template parameter so
// the register indices stay compile-time constants.
template <class F, int RF, class Scale, class Store>
__device__ void forward_from_regs_t(uint32_t* buf, uint32_t log_L, uint32_t log_LW, const uint32_t* twf,
                                    const uint32_t coef[kMaxSetsPerThread][16], Scale scale, Store store) {
  constexpr int R = 1 << RF;
  const uint32_t n_items = (1u << (log_L - RF)) << log_LW;
  const uint32_t log_stride = log_L - (uint32_t)RF;
  const bool single = (uint32_t)RF == log_L;
  __syncthreads();  // shared memory may still be read by the previous phase
#pragma unroll
  for (uint32_t j = 0; j < kMaxSetsPerThread; j++) {
    const uint32_t it = threadIdx.x + j * blockDim.x;
    if (it < n_items) {
      const uint32_t line = it & ((1u << log_LW) - 1u);
      const uint32_t m = it >> log_LW;
      const uint32_t o = bitrev32(m, (int)log_stride);
      uint32_t v[R];
      const uint2 aq = scale(o, line);
      uint32_t cur = aq.x;
#pragma unroll
      for (int k = 0; k < R; k++) {
        v[k] = Fp<F>::mul(coef[j][rev_bits(k, RF)], cur);
        if (k + 1 < R) cur = Fp<F>::mul(cur, aq.y);
      }
      dif_round<F, RF>(v, 0, o, log_L, twf);
#pragma unroll
      for (int k = 0; k < R; k++) {
        const uint32_t pos = o + ((uint32_t)k << log_stride);
        if (single)
          store(pos, line, v[k]);
        else
          buf[sidx(pos, line, log_LW)] = v[k];
      }
    }
  }
  if (single) return;
  __syncthreads();
  uint32_t s0 = (uint32_t)RF;
  while (true) {
    const int r = fwd_round_size(log_L, s0);
    if (s0 + (uint32_t)r == log_L) {
      round_io_r<F>(r, s0, log_L, log_LW, twf,
                    [&](uint32_t pos, uint32_t line) { return buf[sidx(pos, line, log_LW)]; }, store);
      break;
    }
    round_smem_r<F>(r, buf, s0, log_L, log_LW, twf);
    s0 += (uint32_t)r;
    __syncthreads();
  }
}

template <class F, class Scale, class Store>
__device__ __forceinline__ void forward_from_regs(uint32_t* buf, uint32_t log_L, uint32_t log_LW, const uint32_t* twf,
                                                  int r_first, const uint32_t coef[kMaxSetsPerThread][16],
                                                  Scale scale, Store store) {
  switch (r_first) {
    case 1: forward_from_regs_t<F, 1>(buf, log_L, log_LW, twf, coef, scale, store); break;
    case 2: forward_from_regs_t<F, 2>(buf, log_L, log_LW, twf, coef, scale, store); break;
    case 3: forward_from_regs_t<F, 3>(buf, log_L, log_LW, twf, coef, scale, store); break;
    default: forward_from_regs_t<F, 4>(buf, log_L, log_LW, twf, coef, scale, store); break;
  }
}

// Forward DIF with the first round from `load` (pass C).
template <class F, class Load, class Store, class Twist = NoTwist>
__device__ void forward_from_load(uint32_t* buf, uint32_t log_L, uint32_t log_LW, const uint32_t* twf, Load load,
                                  Store store, Twist twist = Twist()) {
  uint32_t s0 = 0;
  bool first = true;
  auto sload = [&](uint32_t pos, uint32_t line) { return buf[sidx(pos, line, log_LW)]; };
  auto sstore = [&](uint32_t pos, uint32_t line, uint32_t v) { buf[sidx(pos, line, log_LW)] = v; };
  while (true) {
    const int r = fwd_round_size(log_L, s0);
    const bool last = s0 + (uint32_t)r == log_L;
    if (first && last)
      round_io_r<F>(r, s0, log_L, log_LW, twf, load, store, twist);
    else if (first)
      round_io_r<F>(r, s0, log_L, log_LW, twf, load, sstore, twist);
    else if (last)
      round_io_r<F>(r, s0, log_L, log_LW, twf, sload, store);
    else
      round_smem_r<F>(r, buf, s0, log_L, log_LW, twf);
    if (last) break;
    first = false;
    s0 += (uint32_t)r;
    __syncthreads();
  }
}

struct TileCtx {
  uint32_t log_L, log_LW, log_ws, ws_mask;
  uint32_t col0, g0;  // first column, first sub-transform of the tile
};

__device__ __forceinline__ TileCtx tile_ctx(const PassGeom& g, uint32_t local) {
  TileCtx t;
  t.log_L = g.log_L;
  t.log_ws = g.log_ws;
  t.log_LW = g.log_ws + g.log_J;
  t.ws_mask = (1u << g.log_ws) - 1u;
  const uint32_t ct = local % g.n_ct;
  const uint32_t grp = (local / g.n_ct) % g.groups;
  t.col0 = ct << g.log_ws;
  t.g0 = grp << g.log_J;
  return t;
}

// Four-step twiddle w_n^(+-s x) on the loads of a first round, s the line's
// sub-transform index and x = o + k * stride the position: {w^(s o), w^(s stride)}.
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

// ---------------------------------------------------------------------------
// One-pass form: tile = all n rows of ws columns.
template <class F>
__global__ void __launch_bounds__(kThreads, 1) k_lde_small(const __grid_constant__ LdeBatch batch,
                                                        const __grid_constant__ TwiddleTables tw) {
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassSmall, blockIdx.x, local);
  const PassGeom g = pass_geom(M, kPassSmall);
  const TileCtx T = tile_ctx(g, local);
  const uint32_t L = 1u << T.log_L, w = M.w;
  const uint32_t* in = M.in;
  if (T.log_L == 0) {
    // height 1: every LDE row equals the input row (the scale g^0 / 1 is 1)
    for (uint32_t line = threadIdx.x; line < (1u << T.log_LW); line += blockDim.x) {
      const uint32_t c = T.col0 + line;
      if (c < w)
        for (uint32_t cb = 0; cb < (1u << M.log_b); cb++) M.out[(uint64_t)cb * w + c] = __ldg(in + c);
    }
    return;
  }
  uint32_t* buf = smem;
  uint32_t* twf = buf + (L << T.log_LW);
  uint32_t* twi = twf + (L >> 1) + 1;
  fill_twiddles<F>(twf, T.log_L, false, tw);
  fill_twiddles<F>(twi, T.log_L, true, tw);
  __syncthreads();
  auto load = [&](uint32_t pos, uint32_t line) -> uint32_t {
    const uint32_t c = T.col0 + line;
    return c < w ? __ldg(in + (uint64_t)pos * w + c) : 0u;
  };
  uint32_t coef[kMaxSetsPerThread][16];
  const int r_last = inverse_to_regs<F>(buf, T.log_L, T.log_LW, twi, load, coef);
  const uint32_t log_stride = T.log_L - (uint32_t)r_last;  // forward first-round stride
  for (uint32_t cb = 0; cb < (1u << M.log_b); cb++) {
    const uint32_t* pt = pw_table(M, cb);
    uint32_t* outb = M.out + (uint64_t)cb * L * w;
    // coefficient i scales by g^i / n, i.e. {g^o / n, g^stride} along a set
    // (table entries carry the 1/n, so the step is multiplied back by n)
    const uint32_t step = Fp<F>::mul(pw_at<F>(pt, 1u << log_stride), n_monty<F>(T.log_L));
    forward_from_regs<F>(
        buf, T.log_L, T.log_LW, twf, r_last, coef,
        [&](uint32_t o, uint32_t) { return make_uint2(pw_at<F>(pt, o), step); },
        [&](uint32_t pos, uint32_t line, uint32_t v) {
          const uint32_t c = T.col0 + line;
          if (c < w) outb[(uint64_t)pos * w + c] = v;
        });
  }
}

// Pass A: rows j2 + n2 * j1 of the input -> T1 rows k1 * n2 + j2 (the
// four-step twiddle w_n^-(j2 k1) is applied by pass B as it loads T1).
template <class F>
__global__ void __launch_bounds__(kThreads, 2) k_lde_a(const __grid_constant__ LdeBatch batch,
                                                       const __grid_constant__ TwiddleTables tw) {
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassA, blockIdx.x, local);
  const PassGeom g = pass_geom(M, kPassA);
  const TileCtx T = tile_ctx(g, local);
  const uint32_t L = 1u << T.log_L, w = M.w, log_n2 = M.log_n2;
  uint32_t* buf = smem;
  uint32_t* twi = buf + (L << T.log_LW);
  fill_twiddles<F>(twi, T.log_L, true, tw);
  __syncthreads();
  auto load = [&](uint32_t pos, uint32_t line) -> uint32_t {
    const uint32_t c = T.col0 + (line & T.ws_mask);
    const uint64_t row = T.g0 + (line >> T.log_ws) + ((uint64_t)pos << log_n2);
    return c < w ? __ldg(M.in + row * w + c) : 0u;
  };
  uint32_t coef[kMaxSetsPerThread][16];
  const int r_last = inverse_to_regs<F>(buf, T.log_L, T.log_LW, twi, load, coef);
  // last-round sets are 16 consecutive positions q, holding frequencies k1 = rev(q)
  const uint32_t n_items = (1u << (T.log_L - r_last)) << T.log_LW;
#pragma unroll
  for (uint32_t j = 0; j < kMaxSetsPerThread; j++) {
    const uint32_t it = threadIdx.x + j * blockDim.x;
    if (it < n_items) {
      const uint32_t line = it & ((1u << T.log_LW) - 1u);
      const uint32_t base = (it >> T.log_LW) << r_last;
      const uint32_t c = T.col0 + (line & T.ws_mask);
      const uint32_t j2 = T.g0 + (line >> T.log_ws);
      if (c < w) {
#pragma unroll
        for (int k = 0; k < 16; k++)
          if (k < (1 << r_last)) {
            const uint32_t k1 = bitrev32(base + (uint32_t)k, (int)T.log_L);
            M.t1[(((uint64_t)k1 << log_n2) + j2) * w + c] = coef[j][k];
          }
      }
    }
  }
}

// Pass B: T1 rows k1 * n2 + j2, times w_n^-(j2 k1) -> coefficients -> per coset
// -> T2 (the twiddle w_n^(k1 k1') is applied by pass C as it loads T2).
template <class F>
__global__ void __launch_bounds__(kThreads, 1) k_lde_b(const __grid_constant__ LdeBatch batch,
                                                       const __grid_constant__ TwiddleTables tw) {
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassB, blockIdx.x, local);
  const PassGeom g = pass_geom(M, kPassB);
  const TileCtx T = tile_ctx(g, local);
  const uint32_t L = 1u << T.log_L, w = M.w, log_n1 = M.log_n1;
  const uint64_t n = 1ull << M.log_n;
  const uint32_t n_mask = (uint32_t)(n - 1);
  uint32_t* buf = smem;
  uint32_t* twf = buf + (L << T.log_LW);
  uint32_t* twi = twf + (L >> 1) + 1;
  fill_twiddles<F>(twf, T.log_L, false, tw);
  fill_twiddles<F>(twi, T.log_L, true, tw);
  __syncthreads();
  auto load = [&](uint32_t pos, uint32_t line) -> uint32_t {
    const uint32_t c = T.col0 + (line & T.ws_mask);
    const uint64_t row = ((uint64_t)(T.g0 + (line >> T.log_ws)) << T.log_L) + pos;
    return c < w ? __ldg(M.t1 + row * w + c) : 0u;
  };
  // element j2 = o + k * stride times w_n^-(k1 j2), k1 the line's sub-transform
  const LineTwist<F, true> twist{&tw, &T, M.log_n, n_mask};
  uint32_t coef[kMaxSetsPerThread][16];
  const int r_last = inverse_to_regs<F>(buf, T.log_L, T.log_LW, twi, load, coef, twist);
  const uint32_t log_stride = T.log_L - (uint32_t)r_last;  // forward first-round stride
  const uint32_t nm = n_monty<F>(M.log_n);
  for (uint32_t cb = 0; cb < (1u << M.log_b); cb++) {
    const uint32_t* pt = pw_table(M, cb);
    // coefficient i = k1 + n1 * p scales by g^i / n: {g^(k1 + n1 o) / n, g^(n1 stride)}
    const uint32_t step = Fp<F>::mul(pw_at<F>(pt, 1u << (log_stride + log_n1)), nm);
    uint32_t* t2 = M.t2 + (uint64_t)cb * n * w;
    forward_from_regs<F>(
        buf, T.log_L, T.log_LW, twf, r_last, coef,
        [&](uint32_t o, uint32_t line) {
          return make_uint2(pw_at<F>(pt, T.g0 + (line >> T.log_ws) + (o << log_n1)), step);
        },
        [&](uint32_t pos, uint32_t line, uint32_t v) {
          const uint32_t c = T.col0 + (line & T.ws_mask);
          if (c < w) {
            const uint32_t k1 = T.g0 + (line >> T.log_ws);
            const uint32_t k1p = bitrev32(pos, (int)T.log_L);
            t2[(((uint64_t)k1p << log_n1) + k1) * w + c] = v;
          }
        });
  }
}

// Pass C: T2 rows cb*n + k1' * n1 + k1 -> out rows cb*n + rev(k1') * n1 + j.
template <class F>
__global__ void __launch_bounds__(kThreads, 2) k_lde_c(const __grid_constant__ LdeBatch batch,
                                                    const __grid_constant__ TwiddleTables tw) {
  extern __shared__ uint32_t smem[];
  uint32_t local;
  const LdeMat& M = find_tile(batch, kPassC, blockIdx.x, local);
  const PassGeom g = pass_geom(M, kPassC);
  const TileCtx T = tile_ctx(g, local);
  const uint32_t L = 1u << T.log_L, w = M.w, log_n2 = M.log_n2;
  const uint32_t cb = local / (g.n_ct * g.groups);
  const uint64_t n = 1ull << M.log_n;
  uint32_t* buf = smem;
  uint32_t* twf = buf + (L << T.log_LW);
  fill_twiddles<F>(twf, T.log_L, false, tw);
  __syncthreads();
  const uint32_t* src = M.t2 + (uint64_t)cb * n * w;
  uint32_t* dst = M.out + (uint64_t)cb * n * w;
  auto load = [&](uint32_t pos, uint32_t line) -> uint32_t {
    const uint32_t c = T.col0 + (line & T.ws_mask);
    const uint64_t row = ((uint64_t)(T.g0 + (line >> T.log_ws)) << T.log_L) + pos;
    return c < w ? __ldg(src + row * w + c) : 0u;
  };
  auto store = [&](uint32_t pos, uint32_t line, uint32_t v) {
    const uint32_t c = T.col0 + (line & T.ws_mask);
    if (c < w) {
      const uint64_t row = ((uint64_t)bitrev32(T.g0 + (line >> T.log_ws), (int)log_n2) << T.log_L) + pos;
      dst[row * w + c] = v;
    }
  };
  // element k1 = o + k * stride times w_n^(k1 k1'), k1' the line's sub-transform
  const LineTwist<F, false> twist{&tw, &T, M.log_n, (uint32_t)(n - 1)};
  forward_from_load<F>(buf, T.log_L, T.log_LW, twf, load, store, twist);
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

void plan_lde_tiling(LdeMat& m) {
  if ((int)m.log_n <= kLdeSmallMaxLog) {
    m.log_n1 = m.log_n2 = 0;
  } else {
    m.log_n1 = (m.log_n + 1) / 2;
    m.log_n2 = m.log_n / 2;
  }
}

// Dynamic shared memory of a pass for one matrix (bytes).
static size_t smem_bytes(const LdeMat& m, int pass) {
  const PassGeom g = pass_geom(m, pass);
  const size_t L = 1ull << g.log_L, LW = 1ull << (g.log_ws + g.log_J);
  const size_t tw_words = (pass == kPassA || pass == kPassC) ? L / 2 + 1 : L + 2;
  return (L * LW + tw_words) * 4;
}

template <class F>
static cudaError_t set_smem_attrs() {
  static std::atomic<uint64_t> done_mask{0};  // one bit per device
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0) return e0;
  const uint64_t bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return cudaSuccess;
  const int cap = 100 * 1024;
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
      for (int ps = 0; ps < 4; ps++) {
        const uint32_t t = lde_tiles(m, ps);
        tiles[ps] += t;
        if (t) sm[ps] = std::max(sm[ps], smem_bytes(m, ps));
      }
    }
    dim3 pgrid((kPwWords << max_b) / 256, batch.n);
    k_pow_tables<F><<<pgrid, 256, 0, st>>>(batch, tw);
    if ((e = cudaGetLastError())) return e;
    if (launches) *launches += 1;
    if (tiles[kPassSmall]) {
      k_lde_small<F><<<tiles[kPassSmall], kThreads, sm[kPassSmall], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      if (launches) *launches += 1;
    }
    if (tiles[kPassA]) {
      k_lde_a<F><<<tiles[kPassA], kThreads, sm[kPassA], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      k_lde_b<F><<<tiles[kPassB], kThreads, sm[kPassB], st>>>(batch, tw);
      if ((e = cudaGetLastError())) return e;
      k_lde_c<F><<<tiles[kPassC], kThreads, sm[kPassC], st>>>(batch, tw);
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
