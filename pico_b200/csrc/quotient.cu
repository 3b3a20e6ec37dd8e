// compute_quotient_values on the GPU (vm/src/machine/utils.rs:201-350).
//
// One thread per point x_i = GENERATOR * w_Q^i of the quotient domain
// (Q = 2^(log_trace + log_qd), natural order i).  The traces are the
// commit's resident LDEs: the quotient domain is the first Q points of the
// LDE domain, so natural point i is committed row rev_Q(i) (the rows
// get_evaluations_on_domain returns, prover.rs:469-489), and the next row is
// point i + 2^log_qd (mod Q).  The chip's constraints come as a straight-line
// register program (pico_constraint_op, see include/pico_gpu.h) that every
// thread runs over its own registers, which live in shared memory laid out
// register-major so a warp's accesses fall on distinct banks.  Each assertion
// folds acc = acc * alpha + c (ProverConstraintFolder::assert_zero /
// assert_zero_ext, vm/src/machine/folder.rs:223-227,321-327); the quotient is
// acc * inv_zerofier.  The Lagrange selectors for the trace domain
// H = <w_n> (shift 1) follow vm/src/compiler/recursion/circuit/domain.rs:48-66:
// Z_H(x) = x^n - 1, is_first_row = Z_H / (x - 1), is_last_row =
// Z_H / (x - w_n^-1), is_transition = x - w_n^-1, inv_zerofier = 1 / Z_H; the
// three inverses share one Fermat inversion per point.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/pico_gpu.h"
#include "field.cuh"
#include "internal.h"
#include "runtime.h"

namespace pico {

constexpr int kQThreads = 128;
constexpr uint32_t kQBaseRegs = 64;  // register file limits of a program
constexpr uint32_t kQExtRegs = 16;

struct QuotientArgs {
  const uint32_t* main;
  const uint32_t* prep;
  const uint32_t* perm;
  uint32_t main_w, prep_w, perm_w;  // words per row (perm: 4 per extension column)
  const uint4* ops;
  uint32_t n_ops;
  const uint32_t* pub;      // public values
  const uint32_t* chal;     // permutation challenges, 4 words each
  const uint32_t* consts;   // regional sum (4), global sum (14), alpha (4)
  uint32_t log_trace, log_qd;
  uint32_t n_base;          // base registers the program uses; the extension registers follow them
  uint32_t chunks;          // 1: point i at out row (i mod D) n + i / D (split_evals order); 0: row i
  uint32_t* out;            // Q x 4
};

template <class F>
__global__ void __launch_bounds__(kQThreads) k_quotient(const __grid_constant__ QuotientArgs A,
                                                         const __grid_constant__ TwiddleTables tw) {
  using B = Fp<F>;
  using E = Ef<F>;
  extern __shared__ uint32_t qsm[];
  uint32_t* rb = qsm + threadIdx.x;                               // base register r at rb[r * kQThreads]
  uint32_t* re = qsm + A.n_base * kQThreads + threadIdx.x;        // ext register r, coeff j at re[(4r+j) * kQThreads]
  const uint32_t log_q = A.log_trace + A.log_qd;
  const uint64_t Q = 1ull << log_q;
  const uint64_t i = (uint64_t)blockIdx.x * kQThreads + threadIdx.x;
  const bool active = i < Q;
  const uint64_t ii = active ? i : 0;
  const uint64_t row_l = bitrev64(ii, (int)log_q);
  const uint64_t row_n = bitrev64((ii + (1ull << A.log_qd)) & (Q - 1), (int)log_q);

  // selectors at x = GENERATOR * w_Q^i
  const uint32_t g = B::to_monty(F::GENERATOR);
  const uint32_t mask = (1u << F::TWO_ADICITY) - 1u;
  const uint32_t e_q = (uint32_t)((ii << (F::TWO_ADICITY - log_q)) & mask);
  const uint32_t x = B::mul(g, B::mul(__ldg(tw.hi + (e_q >> 14)), __ldg(tw.lo + (e_q & 0x3fffu))));
  uint32_t xn = x;
  for (uint32_t k = 0; k < A.log_trace; k++) xn = B::mul(xn, xn);
  const uint32_t e_ninv = (0u - (1u << (F::TWO_ADICITY - A.log_trace))) & mask;  // w_n^-1
  const uint32_t wn_inv = B::mul(__ldg(tw.hi + (e_ninv >> 14)), __ldg(tw.lo + (e_ninv & 0x3fffu)));
  const uint32_t zh = B::sub(xn, F::ONE);
  const uint32_t d1 = B::sub(x, F::ONE), d2 = B::sub(x, wn_inv);
  const uint32_t d12 = B::mul(d1, d2);
  const uint32_t inv = B::inv(B::mul(d12, zh));  // nonzero: the quotient domain is disjoint from H
  const uint32_t inv_zh = B::mul(inv, d12);
  const uint32_t sel_first = B::mul(zh, B::mul(inv, B::mul(d2, zh)));
  const uint32_t sel_last = B::mul(zh, B::mul(inv, B::mul(d1, zh)));
  const uint32_t sel_trans = d2;
  Ext4 alpha, acc{{0, 0, 0, 0}};
#pragma unroll
  for (int j = 0; j < 4; j++) alpha.c[j] = __ldg(A.consts + 18 + j);

  auto ext_get = [&](uint32_t r) {
    Ext4 v;
#pragma unroll
    for (int j = 0; j < 4; j++) v.c[j] = re[(4 * r + j) * kQThreads];
    return v;
  };
  auto ext_set = [&](uint32_t r, const Ext4& v) {
#pragma unroll
    for (int j = 0; j < 4; j++) re[(4 * r + j) * kQThreads] = v.c[j];
  };
  for (uint32_t k = 0; k < A.n_ops; k++) {
    const uint4 o = __ldg(A.ops + k);  // the same instruction for every thread: a broadcast
    const uint32_t d = o.y, a = o.z, b = o.w;
    const uint64_t row = b ? row_n : row_l;
    switch (o.x) {
      case PICO_Q_MAIN: rb[d * kQThreads] = __ldg(A.main + row * A.main_w + a); break;
      case PICO_Q_PREP: rb[d * kQThreads] = __ldg(A.prep + row * A.prep_w + a); break;
      case PICO_Q_PERM: {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(A.perm + row * A.perm_w + 4 * a));
        ext_set(d, Ext4{{v.x, v.y, v.z, v.w}});
        break;
      }
      case PICO_Q_CONST: rb[d * kQThreads] = a; break;
      case PICO_Q_PUBLIC: rb[d * kQThreads] = __ldg(A.pub + a); break;
      case PICO_Q_FIRST: rb[d * kQThreads] = sel_first; break;
      case PICO_Q_LAST: rb[d * kQThreads] = sel_last; break;
      case PICO_Q_TRANSITION: rb[d * kQThreads] = sel_trans; break;
      case PICO_Q_ADD: rb[d * kQThreads] = B::add(rb[a * kQThreads], rb[b * kQThreads]); break;
      case PICO_Q_SUB: rb[d * kQThreads] = B::sub(rb[a * kQThreads], rb[b * kQThreads]); break;
      case PICO_Q_MUL: rb[d * kQThreads] = B::mul(rb[a * kQThreads], rb[b * kQThreads]); break;
      case PICO_Q_EADD: ext_set(d, E::add(ext_get(a), ext_get(b))); break;
      case PICO_Q_ESUB: ext_set(d, E::sub(ext_get(a), ext_get(b))); break;
      case PICO_Q_EMUL: ext_set(d, E::mul(ext_get(a), ext_get(b))); break;
      case PICO_Q_EMB: ext_set(d, Ext4{{rb[a * kQThreads], 0u, 0u, 0u}}); break;
      case PICO_Q_EMULB: ext_set(d, E::scale(ext_get(a), rb[b * kQThreads])); break;
      case PICO_Q_CHALLENGE:
        ext_set(d, Ext4{{__ldg(A.chal + 4 * a), __ldg(A.chal + 4 * a + 1), __ldg(A.chal + 4 * a + 2),
                         __ldg(A.chal + 4 * a + 3)}});
        break;
      case PICO_Q_REGIONAL:
        ext_set(d, Ext4{{__ldg(A.consts), __ldg(A.consts + 1), __ldg(A.consts + 2), __ldg(A.consts + 3)}});
        break;
      case PICO_Q_GLOBAL: rb[d * kQThreads] = __ldg(A.consts + 4 + a); break;
      case PICO_Q_ASSERT: {
        acc = E::mul(acc, alpha);
        acc.c[0] = B::add(acc.c[0], rb[a * kQThreads]);
        break;
      }
      case PICO_Q_EASSERT: acc = E::add(E::mul(acc, alpha), ext_get(a)); break;
      default: break;  // validated on the host
    }
  }
  if (active) {
    const uint4 q = make_uint4(B::mul(acc.c[0], inv_zh), B::mul(acc.c[1], inv_zh), B::mul(acc.c[2], inv_zh),
                               B::mul(acc.c[3], inv_zh));
    const uint64_t orow =
        A.chunks ? ((i & ((1ull << A.log_qd) - 1)) << A.log_trace) + (i >> A.log_qd) : i;  // a permutation of [0, Q)
    reinterpret_cast<uint4*>(A.out)[orow] = q;
  }
}

}  // namespace pico

using namespace pico;

namespace {

// The LDE behind a trace reference, with its checks: a matrix of a resident
// commit of this context and field, tall enough for the quotient domain.
pico_status trace_view(pico_ctx* ctx, const pico_trace_ref& r, int field, uint32_t log_q, const char* what,
                       bool required, const uint32_t** ptr, uint32_t* width) {
  *ptr = nullptr;
  *width = 0;
  if (!r.commit) {
    if (required) {
      set_error("quotient_values: the %s trace is required", what);
      return PICO_ERR_INVALID_ARG;
    }
    return PICO_OK;
  }
  const pico_commit* c = r.commit;
  if (c->ctx != ctx || c->field != field || r.mat_idx >= c->n_mats) {
    set_error("quotient_values: the %s trace is not a matrix of a commit of this context and field", what);
    return PICO_ERR_INVALID_ARG;
  }
  if (c->shard_log) {
    set_error("quotient_values: the %s trace's commitment is one shard of a row-split commit", what);
    return PICO_ERR_UNSUPPORTED;
  }
  if (c->log_N[r.mat_idx] < log_q) {
    set_error("quotient_values: the %s LDE has 2^%u rows, fewer than the quotient domain's 2^%u", what,
              c->log_N[r.mat_idx], log_q);
    return PICO_ERR_INVALID_ARG;
  }
  *ptr = c->lde[r.mat_idx];
  *width = c->width[r.mat_idx];
  return PICO_OK;
}

}  // namespace

extern "C" pico_status pico_gpu_quotient_values(pico_ctx* ctx, pico_trace_ref preprocessed, pico_trace_ref main,
                                                pico_trace_ref permutation, uint32_t log_trace_height,
                                                uint32_t log_quotient_degree, const pico_constraint_op* program,
                                                uint32_t n_ops, const uint32_t* public_values, uint32_t n_public,
                                                const uint32_t* perm_challenges, uint32_t n_challenges,
                                                const uint32_t regional_sum[4], const uint32_t global_sum[14],
                                                const uint32_t alpha[4], uint32_t* out, uint32_t flags) {
  if (!ctx || !main.commit || (!program && n_ops) || !alpha || !out || (n_public && !public_values) ||
      (n_challenges && !perm_challenges)) {
    set_error("quotient_values: null argument");
    return PICO_ERR_INVALID_ARG;
  }
  if (flags & ~(PICO_OUTPUT_DEVICE | PICO_QUOTIENT_CHUNKS)) {
    set_error("quotient_values: unknown flags 0x%x", flags);
    return PICO_ERR_INVALID_ARG;
  }
  const int field = main.commit->field;
  const uint32_t S = field == PICO_KOALABEAR ? 24u : 27u;
  const uint32_t log_q = log_trace_height + log_quotient_degree;
  if (log_trace_height == 0 || log_q > S || log_quotient_degree > kLdeMaxLogBlowup) {
    set_error("quotient_values: trace 2^%u with quotient degree 2^%u is not supported", log_trace_height,
              log_quotient_degree);
    return PICO_ERR_INVALID_ARG;
  }
  pico_status s;
  const uint32_t *pm, *pp, *pe;
  uint32_t wm, wp, we;
  if ((s = trace_view(ctx, main, field, log_q, "main", true, &pm, &wm)) ||
      (s = trace_view(ctx, preprocessed, field, log_q, "preprocessed", false, &pp, &wp)) ||
      (s = trace_view(ctx, permutation, field, log_q, "permutation", false, &pe, &we)))
    return s;
  if (we % 4) {
    set_error("quotient_values: the permutation trace has %u words per row, not whole extension elements", we);
    return PICO_ERR_INVALID_ARG;
  }
  // the program: every register, column and table index in range; the
  // register files are sized to the highest register it names, so a small
  // program leaves shared memory for more resident CTAs
  uint32_t n_base = 1, n_ext = 1;
  for (uint32_t k = 0; k < n_ops; k++) {
    const pico_constraint_op& o = program[k];
    bool ok;
    const bool db = o.dst < kQBaseRegs, de = o.dst < kQExtRegs;
    switch (o.op) {
      case PICO_Q_MAIN: ok = db && o.a < wm && o.b <= 1; break;
      case PICO_Q_PREP: ok = db && pp && o.a < wp && o.b <= 1; break;
      case PICO_Q_PERM: ok = de && pe && o.a < we / 4 && o.b <= 1; break;
      case PICO_Q_CONST: ok = db && o.a < (field == PICO_KOALABEAR ? KoalaBear::P : BabyBear::P); break;
      case PICO_Q_PUBLIC: ok = db && o.a < n_public; break;
      case PICO_Q_FIRST: case PICO_Q_LAST: case PICO_Q_TRANSITION: ok = db; break;
      case PICO_Q_ADD: case PICO_Q_SUB: case PICO_Q_MUL: ok = db && o.a < kQBaseRegs && o.b < kQBaseRegs; break;
      case PICO_Q_EADD: case PICO_Q_ESUB: case PICO_Q_EMUL: ok = de && o.a < kQExtRegs && o.b < kQExtRegs; break;
      case PICO_Q_EMB: ok = de && o.a < kQBaseRegs; break;
      case PICO_Q_EMULB: ok = de && o.a < kQExtRegs && o.b < kQBaseRegs; break;
      case PICO_Q_CHALLENGE: ok = de && o.a < n_challenges; break;
      case PICO_Q_REGIONAL: ok = de && regional_sum; break;
      case PICO_Q_GLOBAL: ok = db && o.a < 14 && global_sum; break;
      case PICO_Q_ASSERT: ok = o.a < kQBaseRegs; break;
      case PICO_Q_EASSERT: ok = o.a < kQExtRegs; break;
      default: ok = false;
    }
    if (!ok) {
      set_error("quotient_values: program instruction %u (op %u, dst %u, a %u, b %u) is out of range", k, o.op,
                o.dst, o.a, o.b);
      return PICO_ERR_INVALID_ARG;
    }
    // registers named (in range, checked above): which operands are base or extension registers
    auto base = [&](uint32_t r) { n_base = std::max(n_base, r + 1); };
    auto ext = [&](uint32_t r) { n_ext = std::max(n_ext, r + 1); };
    switch (o.op) {
      case PICO_Q_MAIN: case PICO_Q_PREP: case PICO_Q_CONST: case PICO_Q_PUBLIC: case PICO_Q_FIRST:
      case PICO_Q_LAST: case PICO_Q_TRANSITION: case PICO_Q_GLOBAL: base(o.dst); break;
      case PICO_Q_ADD: case PICO_Q_SUB: case PICO_Q_MUL: base(o.dst); base(o.a); base(o.b); break;
      case PICO_Q_PERM: case PICO_Q_CHALLENGE: case PICO_Q_REGIONAL: ext(o.dst); break;
      case PICO_Q_EADD: case PICO_Q_ESUB: case PICO_Q_EMUL: ext(o.dst); ext(o.a); ext(o.b); break;
      case PICO_Q_EMB: ext(o.dst); base(o.a); break;
      case PICO_Q_EMULB: ext(o.dst); ext(o.a); base(o.b); break;
      case PICO_Q_ASSERT: base(o.a); break;
      case PICO_Q_EASSERT: ext(o.a); break;
      default: break;
    }
  }
  const size_t smem = (size_t)(n_base + 4 * n_ext) * kQThreads * 4;  // at most 64 KiB
  const uint64_t Q = 1ull << log_q;
  const bool out_dev = flags & PICO_OUTPUT_DEVICE;
  // one device block: program, public values, challenges, constants, then the output if on the host
  const uint64_t w_ops = 4ull * n_ops, w_pub = n_public, w_chal = 4ull * n_challenges, w_const = 22;
  const uint64_t w_in = w_ops + w_pub + w_chal + w_const;
  const uint64_t off_out = (w_in + 63) & ~63ull;
  const uint64_t bytes = 4 * (off_out + (out_dev ? 0 : 4 * Q));
  if (!try_reserve(ctx, bytes)) {
    set_error("quotient_values: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = pick_stream(ctx);
  uint32_t* blk = nullptr;
  if ((s = device_alloc((void**)&blk, bytes, st))) {
    unreserve(ctx, bytes);
    return s;
  }
  std::vector<uint32_t> host(w_in, 0);
  if (n_ops) memcpy(host.data(), program, 16ull * n_ops);
  if (n_public) memcpy(host.data() + w_ops, public_values, 4ull * n_public);
  if (n_challenges) memcpy(host.data() + w_ops + w_pub, perm_challenges, 16ull * n_challenges);
  uint32_t* cst = host.data() + w_ops + w_pub + w_chal;
  if (regional_sum) memcpy(cst, regional_sum, 16);
  if (global_sum) memcpy(cst + 4, global_sum, 56);
  memcpy(cst + 18, alpha, 16);
  s = cuda_status(cudaMemcpyAsync(blk, host.data(), 4 * w_in, cudaMemcpyHostToDevice, st), "program upload");
  QuotientArgs A;
  A.main = pm;
  A.prep = pp;
  A.perm = pe;
  A.main_w = wm;
  A.prep_w = wp;
  A.perm_w = we;
  A.ops = reinterpret_cast<const uint4*>(blk);
  A.n_ops = n_ops;
  A.pub = blk + w_ops;
  A.chal = blk + w_ops + w_pub;
  A.consts = blk + w_ops + w_pub + w_chal;
  A.log_trace = log_trace_height;
  A.log_qd = log_quotient_degree;
  A.n_base = n_base;
  A.chunks = (flags & PICO_QUOTIENT_CHUNKS) ? 1u : 0u;
  A.out = out_dev ? out : blk + off_out;
  const TwiddleTables tw = twiddles(ctx, field);
  const unsigned grid = (unsigned)((Q + kQThreads - 1) / kQThreads);
  if (!s) {
    cudaError_t e;
    if (field == PICO_KOALABEAR) {
      e = cudaFuncSetAttribute(k_quotient<KoalaBear>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (!e) k_quotient<KoalaBear><<<grid, kQThreads, smem, st>>>(A, tw);
    } else {
      e = cudaFuncSetAttribute(k_quotient<BabyBear>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (!e) k_quotient<BabyBear><<<grid, kQThreads, smem, st>>>(A, tw);
    }
    s = cuda_status(e ? e : cudaGetLastError(), "quotient kernel");
  }
  if (!s && !out_dev)
    s = cuda_status(cudaMemcpyAsync(out, blk + off_out, 16 * Q, cudaMemcpyDeviceToHost, st), "quotient read-back");
  cudaFreeAsync(blk, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "quotient_values");
  unreserve(ctx, bytes);
  return s ? s : s2;
}
