// FRI commit phase on device-resident codewords (the loop inside
// TwoAdicFriPcs::open, prover.rs:589; mirrored by the verifier's
// verify_shape_and_sample_challenges, vm/src/compiler/recursion/circuit/fri.rs:45-52).
//
// Every round runs on one stream with no host round trip: leaf hashing of the
// codeword viewed as a (len/2) x 8 base matrix (ExtensionMmcs flattening, one
// permutation per leaf), compression up to the root, the duplex challenger
// observing the root and sampling beta on the device, then the fold.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "internal.h"
#include "runtime.h"

using namespace pico;

namespace pico {
pico_status enqueue_fri_rounds(int field, cudaStream_t st, const TwiddleTables& tw, uint32_t log_n, uint32_t R,
                               const std::vector<uint32_t*>& codewords, const std::vector<uint32_t*>& trees,
                               uint32_t* d_betas, DevChallenger* d_ch, const uint32_t* const* inject,
                               uint32_t* launches) {
  pico_status s;
  uint32_t nl = 0;
  for (uint32_t r = 0; r < R; r++) {
    const uint32_t L = log_n - r;            // codeword length 2^L
    const uint64_t leaves = 1ull << (L - 1);  // rows of the (len/2) x 8 matrix
    if (r == 0) {
      // later rounds' leaves come out of the previous round's fold
      RowGroup g;
      memset(&g, 0, sizeof g);
      g.n_segs = 1;
      g.total_width = 8;
      g.segs[0].ptr = codewords[0];
      g.segs[0].width = 8;
      if ((s = cuda_status(launch_hash_rows(field, g, leaves, trees[0], st), "FRI leaf hashing"))) return s;
      nl++;
    }
    // wide levels one launch each; from 2^15 nodes down, seven levels per
    // launch (k_subtree_quad); the last <= 512 nodes and the challenger in
    // one block
    uint32_t* layer = trees[r];
    uint64_t n = leaves;
    while (n > 512) {
      if (n <= (1u << 15)) {
        if ((s = cuda_status(launch_subtree(field, layer, (uint32_t)n, SubtreeInj{}, st), "FRI subtree"))) return s;
        nl++;
        for (int l = 0; l < 7; l++) {
          layer += n * 8;
          n /= 2;
        }
        continue;
      }
      uint32_t* next = layer + n * 8;
      if ((s = cuda_status(launch_compress(field, layer, next, n / 2, nullptr, st), "FRI compression"))) return s;
      nl++;
      layer = next;
      n /= 2;
    }
    if ((s = cuda_status(launch_tree_top(field, layer, (uint32_t)n, d_ch, d_betas + 4 * r, st), "FRI tree top")))
      return s;
    nl++;
    const uint32_t* inj = inject ? inject[r] : nullptr;
    if (r + 1 < R)
      s = cuda_status(launch_fri_fold_hash(field, codewords[r], L, d_betas + 4 * r, tw, codewords[r + 1], inj,
                                           trees[r + 1], st),
                      "fold and hash");
    else
      s = cuda_status(launch_fri_fold_tw(field, codewords[r], L, d_betas + 4 * r, tw, codewords[r + 1], st, inj),
                      "fold");
    if (s) return s;
    nl++;
  }
  if (launches) *launches = nl;
  return PICO_OK;
}
}  // namespace pico

static pico_status fri_alloc(void** p, size_t bytes, cudaStream_t st) {
  return cuda_status(cudaMallocAsync(p, bytes ? bytes : 16, st), "device allocation");
}

extern "C" pico_status pico_gpu_fri_commit_phase(pico_ctx* ctx, pico_field field, const uint32_t* codeword,
                                                 uint32_t log_n, uint32_t log_blowup, uint32_t log_final_len,
                                                 const uint32_t* betas_in, pico_challenger* ch, uint32_t flags,
                                                 uint32_t* roots, uint32_t* betas, uint32_t* final_out,
                                                 uint32_t* n_rounds, pico_fri** out) {
  if (out) *out = nullptr;
  if (!ctx || !codeword || (field != PICO_KOALABEAR && field != PICO_BABYBEAR)) {
    set_error("fri_commit_phase: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t S = field == PICO_KOALABEAR ? 24u : 27u;
  const uint32_t log_stop = log_blowup + log_final_len;
  if (log_n > S || log_n < log_stop || log_n < 1) {
    set_error("fri_commit_phase: codeword 2^%u vs stop length 2^%u (two-adicity %u)", log_n, log_stop, S);
    return PICO_ERR_INVALID_ARG;
  }
  if (!betas_in && !ch) {
    set_error("fri_commit_phase: need a challenger state or explicit betas");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t R = log_n - log_stop;
  // Footprint: all codewords, all trees, small buffers.
  uint64_t resident = 0;
  for (uint32_t r = 0; r <= R; r++) resident += (16ull << (log_n - r));
  for (uint32_t r = 0; r < R; r++) resident += ((2ull << (log_n - r - 1)) - 1) * 32;
  resident += 256ull * (2 * R + 1);  // alignment of the views into one block
  const uint64_t small = 4096 + 16ull * (R + 1) + (16ull << log_final_len);
  if (!try_reserve(ctx, resident + small)) {
    set_error("fri_commit_phase: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  cudaSetDevice(ctx->device);
  uint32_t slot = 0;
  cudaStream_t st = pick_stream(ctx, nullptr, &slot);
  auto f = std::make_unique<pico_fri>();
  f->ctx = ctx;
  f->field = field;
  f->log_n = log_n;
  f->rounds = R;
  f->bytes_resident = resident;
  std::vector<void*> scratch;
  std::vector<uint32_t> final_cw(4u << log_stop);
  uint32_t err_flag = 0;
  const TwiddleTables tw = twiddles(ctx, field);

  auto run = [&]() -> pico_status {
    pico_status s;
    void* p;
    // codewords and trees: one block (views at 256-byte aligned offsets);
    // one stream-ordered allocation per round would cost more host time than
    // the small rounds take on the device
    uint64_t bytes = 0;
    std::vector<uint64_t> off_cw(R + 1), off_tree(R);
    auto take = [&](uint64_t b) {
      const uint64_t o = bytes;
      bytes += (b + 255) & ~255ull;
      return o;
    };
    for (uint32_t r = 0; r <= R; r++) off_cw[r] = take(16ull << (log_n - r));
    for (uint32_t r = 0; r < R; r++) off_tree[r] = take(((2ull << (log_n - r - 1)) - 1) * 32);
    if ((s = fri_alloc(&p, bytes, st))) return s;
    f->arena = p;
    for (uint32_t r = 0; r <= R; r++) f->codewords.push_back((uint32_t*)((uint8_t*)p + off_cw[r]));
    for (uint32_t r = 0; r < R; r++) f->trees.push_back((uint32_t*)((uint8_t*)p + off_tree[r]));
    if ((s = cuda_status(cudaMemcpyAsync(f->codewords[0], codeword, 16ull << log_n,
                                         (flags & PICO_INPUT_DEVICE) ? cudaMemcpyDeviceToDevice
                                                                     : cudaMemcpyHostToDevice,
                                         st),
                         "codeword copy")))
      return s;
    // betas, error flag, final polynomial and challenger: one scratch block
    const uint64_t b_betas = (16ull * (R + 1) + 255) & ~255ull, b_err = 256;
    const uint64_t b_final = ((16ull << log_final_len) + 255) & ~255ull;
    if ((s = fri_alloc(&p, b_betas + b_err + b_final + sizeof(DevChallenger), st))) return s;
    scratch.push_back(p);
    uint32_t* d_betas = (uint32_t*)p;
    uint32_t* d_err = (uint32_t*)((uint8_t*)p + b_betas);
    uint32_t* d_final = (uint32_t*)((uint8_t*)p + b_betas + b_err);
    DevChallenger* d_ch = nullptr;
    if ((s = cuda_status(cudaMemsetAsync(d_err, 0, 4, st), "memset"))) return s;
    if (betas_in) {
      if ((s = cuda_status(cudaMemcpyAsync(d_betas, betas_in, 16ull * R, cudaMemcpyHostToDevice, st), "betas")))
        return s;
    }
    if (ch) {
      static_assert(sizeof(DevChallenger) == sizeof(pico_challenger), "challenger layout");
      d_ch = (DevChallenger*)((uint8_t*)scratch.back() + b_betas + b_err + b_final);
      if ((s = cuda_status(cudaMemcpyAsync(d_ch, ch, sizeof *ch, cudaMemcpyHostToDevice, st), "challenger")))
        return s;
    }
    if ((s = enqueue_fri_rounds(field, st, tw, log_n, R, f->codewords, f->trees, d_betas, betas_in ? nullptr : d_ch,
                                nullptr, nullptr)))
      return s;
    // Read-backs are queued after the whole loop: a copy into pageable host
    // memory blocks the calling thread until the stream reaches it.
    uint32_t* last = f->codewords[R];
    if (log_final_len == 0) {
      if (!betas_in)
        if ((s = cuda_status(launch_challenger_observe(field, d_ch, last, 4, st), "observe final"))) return s;
    } else {
      if ((s = cuda_status(launch_fri_final_poly(field, last, log_stop, log_final_len, tw, d_final, d_err, st),
                           "final polynomial")))
        return s;
      if (!betas_in)
        if ((s = cuda_status(launch_challenger_observe(field, d_ch, d_final, 4u << log_final_len, st),
                             "observe final")))
          return s;
      if (final_out)
        if ((s = cuda_status(cudaMemcpyAsync(final_out, d_final, 16ull << log_final_len, cudaMemcpyDeviceToHost, st),
                             "final copy")))
          return s;
    }
    if ((s = cuda_status(cudaMemcpyAsync(final_cw.data(), last, 16ull << log_stop, cudaMemcpyDeviceToHost, st),
                         "final codeword")))
      return s;
    if ((s = cuda_status(cudaMemcpyAsync(&err_flag, d_err, 4, cudaMemcpyDeviceToHost, st), "flag"))) return s;
    if (roots)
      for (uint32_t r = 0; r < R; r++) {
        // the root is the last digest of round r's tree
        const uint64_t leaves = 1ull << (log_n - r - 1);
        if ((s = cuda_status(cudaMemcpyAsync(roots + 8 * r, f->trees[r] + (2 * leaves - 2) * 8, 32,
                                             cudaMemcpyDeviceToHost, st),
                             "root copy")))
          return s;
      }
    if (betas && R)
      if ((s = cuda_status(cudaMemcpyAsync(betas, d_betas, 16ull * R, cudaMemcpyDeviceToHost, st), "betas copy")))
        return s;
    if (ch && !betas_in)
      if ((s = cuda_status(cudaMemcpyAsync(ch, d_ch, sizeof *ch, cudaMemcpyDeviceToHost, st), "challenger copy")))
        return s;
    return PICO_OK;
  };
  pico_status s = run();
  for (void* p : scratch) cudaFreeAsync(p, st);
  if (!s) s = guard_enqueue(ctx, slot, st);
  pico_status s2 = cuda_status(cudaStreamSynchronize(st), "fri_commit_phase");
  if (!s) s = s2;
  if (!s) s = guard_verdict(ctx, slot);
  unreserve(ctx, small);
  if (!s && log_final_len == 0) {
    // Plonky3 asserts the remaining 2^b evaluations of the constant polynomial agree.
    for (size_t i = 1; i < (size_t)1 << log_stop; i++)
      if (memcmp(&final_cw[4 * i], &final_cw[0], 16) != 0) {
        set_error("fri_commit_phase: final codeword is not constant (input is not of low degree)");
        s = PICO_ERR_INVALID_ARG;
        break;
      }
    if (!s && final_out) memcpy(final_out, final_cw.data(), 16);
  }
  if (!s && err_flag) {
    set_error("fri_commit_phase: final polynomial has more than 2^%u coefficients", log_final_len);
    s = PICO_ERR_INVALID_ARG;
  }
  if (!s && n_rounds) *n_rounds = R;
  if (s || !out) {
    if (f->arena) cudaFreeAsync(f->arena, st);
    cudaStreamSynchronize(st);
    unreserve(ctx, resident);
    return s;
  }
  *out = f.release();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_fri_release(pico_ctx* ctx, pico_fri* f) {
  if (!f) return PICO_OK;
  if (!ctx || f->ctx != ctx) {
    set_error("fri_release: handle belongs to another context");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = aux_stream(ctx);
  if (f->arena) cudaFreeAsync(f->arena, st);
  pico_status s = cuda_status(cudaStreamSynchronize(st), "fri_release");
  unreserve(ctx, f->bytes_resident);
  delete f;
  return s;
}

extern "C" pico_status pico_gpu_fri_layer(pico_ctx* ctx, const pico_fri* f, uint32_t round, uint32_t* out,
                                          uint32_t flags) {
  if (!ctx || !f || !out || round > f->rounds) {
    set_error("fri_layer: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t st = aux_stream(ctx);
  pico_status s = cuda_status(cudaMemcpyAsync(out, f->codewords[round], 16ull << (f->log_n - round),
                                              (flags & PICO_OUTPUT_DEVICE) ? cudaMemcpyDeviceToDevice
                                                                           : cudaMemcpyDeviceToHost,
                                              st),
                              "fri_layer copy");
  if (s) return s;
  return cuda_status(cudaStreamSynchronize(st), "fri_layer");
}

// ---------------------------------------------------------------------------
// The FRI commit phase of a codeword split by rows over 2^k devices (the row
// partition of pico_gpu_commit_shard).  A round's tree is MerkleTreeMmcs over
// the codeword viewed as (len/2) x 8 base words: leaf i is rows 2i, 2i + 1, so
// shard s's rows make the subtree under node s at depth k.  The fold pairs the
// same rows, so the next codeword's shard s rows are the fold of this shard's
// rows: nothing crosses devices but the 8-word shard roots (and the final
// gather of a short codeword, done by the caller).

struct pico_fri_shard {
  pico_ctx* ctx = nullptr;
  int field = 0;
  uint32_t log_len = 0;     // the whole codeword of the current round: 2^log_len rows
  uint32_t log_shards = 0, shard = 0;
  uint32_t* cw[2] = {nullptr, nullptr};  // this shard's rows of the current / next codeword
  uint32_t cur = 0;
  uint32_t* tree = nullptr;  // digest layers of the current round's subtree, leaves first
  uint32_t* d_beta = nullptr;
  void* block = nullptr;
  uint64_t bytes = 0;
  cudaStream_t st = nullptr;
  uint32_t slot = 0;
  uint32_t log_rows() const { return log_len - log_shards; }
};

namespace {

// Compression levels of the current subtree (its leaves in fs->tree) up to its
// root, then the root to the host.
pico_status shard_tree_root(pico_fri_shard* fs, uint32_t root[8]) {
  pico_status s;
  const uint64_t leaves = 1ull << (fs->log_rows() - 1);
  uint32_t* layer = fs->tree;
  uint64_t n = leaves;
  while (n > 512) {
    if (n <= (1u << 15)) {
      if ((s = cuda_status(launch_subtree(fs->field, layer, (uint32_t)n, SubtreeInj{}, fs->st), "FRI subtree")))
        return s;
      for (int l = 0; l < 7; l++) {
        layer += n * 8;
        n /= 2;
      }
      continue;
    }
    uint32_t* next = layer + n * 8;
    if ((s = cuda_status(launch_compress(fs->field, layer, next, n / 2, nullptr, fs->st), "FRI compression")))
      return s;
    layer = next;
    n /= 2;
  }
  if ((s = cuda_status(launch_tree_top(fs->field, layer, (uint32_t)n, nullptr, nullptr, fs->st), "FRI tree top")))
    return s;
  if ((s = cuda_status(cudaMemcpyAsync(root, fs->tree + (2 * leaves - 2) * 8, 32, cudaMemcpyDeviceToHost, fs->st),
                       "root copy")))
    return s;
  if ((s = guard_enqueue(fs->ctx, fs->slot, fs->st))) return s;
  if ((s = cuda_status(cudaStreamSynchronize(fs->st), "FRI shard round"))) return s;
  return guard_verdict(fs->ctx, fs->slot);
}

}  // namespace

extern "C" pico_status pico_gpu_fri_shard_begin(pico_ctx* ctx, pico_field field, const uint32_t* rows,
                                                uint32_t log_n, uint32_t log_shards, uint32_t shard,
                                                uint32_t flags, pico_fri_shard** out, uint32_t root[8]) {
  if (out) *out = nullptr;
  if (!ctx || !rows || !out || !root || (field != PICO_KOALABEAR && field != PICO_BABYBEAR)) {
    set_error("fri_shard_begin: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  const uint32_t S = field == PICO_KOALABEAR ? 24u : 27u;
  if (log_n > S || log_shards > 20 || log_n < log_shards + 1 || shard >= (1u << log_shards)) {
    set_error("fri_shard_begin: codeword 2^%u in 2^%u shards (shard %u): each shard needs two rows", log_n,
              log_shards, shard);
    return PICO_ERR_INVALID_ARG;
  }
  if (flags & ~PICO_INPUT_DEVICE) {
    set_error("fri_shard_begin: unknown flags 0x%x", flags);
    return PICO_ERR_INVALID_ARG;
  }
  auto fs = std::make_unique<pico_fri_shard>();
  fs->ctx = ctx;
  fs->field = field;
  fs->log_len = log_n;
  fs->log_shards = log_shards;
  fs->shard = shard;
  const uint32_t lr = log_n - log_shards;
  const uint64_t b0 = ((16ull << lr) + 255) & ~255ull, b1 = ((16ull << (lr - 1)) + 255) & ~255ull;
  const uint64_t bt = ((((2ull << (lr - 1)) - 1) * 32) + 255) & ~255ull;
  fs->bytes = b0 + b1 + bt + 256;
  if (!try_reserve(ctx, fs->bytes)) {
    set_error("fri_shard_begin: HBM budget exceeded");
    return PICO_ERR_OUT_OF_MEMORY;
  }
  cudaSetDevice(ctx->device);
  fs->st = pick_stream(ctx, nullptr, &fs->slot);
  pico_status s = device_alloc(&fs->block, fs->bytes, fs->st);
  if (s) {
    unreserve(ctx, fs->bytes);
    return s;
  }
  uint8_t* p = (uint8_t*)fs->block;
  fs->cw[0] = (uint32_t*)p;
  fs->cw[1] = (uint32_t*)(p + b0);
  fs->tree = (uint32_t*)(p + b0 + b1);
  fs->d_beta = (uint32_t*)(p + b0 + b1 + bt);
  // round 0: this shard's rows, their leaves (one permutation per row pair) and subtree
  RowGroup g;
  memset(&g, 0, sizeof g);
  g.n_segs = 1;
  g.total_width = 8;
  g.segs[0].ptr = fs->cw[0];
  g.segs[0].width = 8;
  s = cuda_status(cudaMemcpyAsync(fs->cw[0], rows, 16ull << lr,
                                  (flags & PICO_INPUT_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  fs->st),
                  "codeword rows");
  if (!s) s = cuda_status(launch_hash_rows(field, g, 1ull << (lr - 1), fs->tree, fs->st), "FRI leaf hashing");
  if (!s) s = shard_tree_root(fs.get(), root);
  if (s) {
    cudaStreamSynchronize(fs->st);
    cudaFreeAsync(fs->block, fs->st);
    cudaStreamSynchronize(fs->st);
    unreserve(ctx, fs->bytes);
    return s;
  }
  *out = fs.release();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_fri_shard_fold(pico_fri_shard* fs, const uint32_t beta[4], uint32_t root[8]) {
  if (!fs || !beta || !root) {
    set_error("fri_shard_fold: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  if (fs->log_rows() < 2) {
    set_error("fri_shard_fold: the shard holds 2^%u rows, too few to fold into a tree; gather the codeword",
              fs->log_rows());
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(fs->ctx->device);
  pico_status s;
  if ((s = cuda_status(cudaMemcpyAsync(fs->d_beta, beta, 16, cudaMemcpyHostToDevice, fs->st), "beta"))) return s;
  const uint64_t new_rows = 1ull << (fs->log_rows() - 1);
  if ((s = cuda_status(launch_fri_fold_hash_rows(fs->field, fs->cw[fs->cur], fs->log_len, fs->shard * new_rows,
                                                 new_rows / 2, fs->d_beta, twiddles(fs->ctx, fs->field),
                                                 fs->cw[fs->cur ^ 1], fs->tree, fs->st),
                       "shard fold and hash")))
    return s;
  fs->cur ^= 1;
  fs->log_len--;
  return shard_tree_root(fs, root);
}

extern "C" pico_status pico_gpu_fri_shard_rows(pico_fri_shard* fs, uint32_t* out, uint32_t flags) {
  if (!fs || !out || (flags & ~PICO_OUTPUT_DEVICE)) {
    set_error("fri_shard_rows: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  cudaSetDevice(fs->ctx->device);
  pico_status s = cuda_status(cudaMemcpyAsync(out, fs->cw[fs->cur], 16ull << fs->log_rows(),
                                              (flags & PICO_OUTPUT_DEVICE) ? cudaMemcpyDeviceToDevice
                                                                           : cudaMemcpyDeviceToHost,
                                              fs->st),
                              "shard rows");
  if (s) return s;
  return cuda_status(cudaStreamSynchronize(fs->st), "fri_shard_rows");
}

extern "C" pico_status pico_gpu_fri_shard_release(pico_fri_shard* fs) {
  if (!fs) return PICO_OK;
  cudaSetDevice(fs->ctx->device);
  cudaFreeAsync(fs->block, fs->st);
  pico_status s = cuda_status(cudaStreamSynchronize(fs->st), "fri_shard_release");
  unreserve(fs->ctx, fs->bytes);
  delete fs;
  return s;
}
