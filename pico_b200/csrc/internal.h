// Internal host-side interface between the C-ABI runtime (api.cu) and the
// kernel translation units.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pico {

constexpr int kMaxSegs = 64;  // matrices concatenated into one Merkle row

// One matrix segment of a concatenated Merkle row: `rows` x `width`,
// row-major, rows at ptr + r * width.
struct RowSeg {
  const uint32_t* ptr;
  uint32_t width;
  uint32_t pad;
};

// Rows of all matrices of one height, concatenated in commit order (the
// MerkleTreeMmcs leaf / injection input, fri.rs:389-436).
struct RowGroup {
  uint32_t n_segs;
  uint32_t total_width;
  RowSeg segs[kMaxSegs];
};

// --- Poseidon2 / Merkle kernels (p2_kernels.cu) -------------------------
cudaError_t upload_p2_constants(int field, const uint32_t ext[8][16], const uint32_t* inte, int rounds_p,
                                const uint32_t diag[16]);
// four_lanes: four threads per state (the latency form).
cudaError_t launch_permute(int field, uint32_t* states, uint64_t n, cudaStream_t st, bool four_lanes = false);
// Levels of at most this many nodes are compressed four threads per node.
constexpr uint64_t kQuadMaxNodes = 16384;
cudaError_t launch_hash_rows(int field, const RowGroup& g, uint64_t rows, uint32_t* out, cudaStream_t st,
                             unsigned block = 256);
// Row digests of several height groups in one launch.  Group g owns global
// rows [row_end[g-1], row_end[g]) (row_end[-1] = 0), its row r is the
// concatenation of segs[seg_begin[g] .. seg_begin[g+1]) and its digest goes to
// out[g] + 8 r.
constexpr int kBatchGroups = 16;
constexpr int kBatchSegs = 128;
struct GroupBatch {
  uint32_t n_groups;
  uint32_t n_segs;
  uint64_t row_end[kBatchGroups];
  uint32_t* out[kBatchGroups];
  uint32_t seg_begin[kBatchGroups + 1];
  uint32_t width[kBatchGroups];
  RowSeg segs[kBatchSegs];
};
cudaError_t launch_hash_groups(int field, const GroupBatch& b, cudaStream_t st, unsigned block = 256);
// Resumable row sponge: continue from state_in (nullptr: zero state) at rate
// position pos0; if digest_out, finish and write 8-word digests, else store
// the 16-word states to state_out.  Row r's state is 16 consecutive words.
cudaError_t launch_absorb_rows(int field, const RowGroup& g, uint64_t rows, uint32_t pos0, const uint32_t* state_in,
                               uint32_t* state_out, uint32_t* digest_out, cudaStream_t st, unsigned block = 256);
// Seven levels at once: a level of n_in nodes (a multiple of 128) down to
// n_in / 128, every level written after the previous one (tree layout).
constexpr uint32_t kSubtreeIn = 128;  // input nodes per CTA (seven levels down to one)
struct SubtreeInj {
  const uint32_t* digests[7];  // per computed level (nullptr: none), 8 words per node
};
cudaError_t launch_subtree(int field, uint32_t* level, uint32_t n_in, const SubtreeInj& inj, cudaStream_t st);
// next[i] = compress(prev[2i], prev[2i+1]); if inj_digests != null:
// next[i] = compress(next[i], inj_digests[i]) (8 words per digest).
cudaError_t launch_compress(int field, const uint32_t* prev, uint32_t* next, uint64_t n_next,
                            const uint32_t* inj_digests, cudaStream_t st);

// --- FRI kernels (p2_kernels.cu) ----------------------------------------
// Device-side duplex challenger state, Monty form.
struct DevChallenger {
  uint32_t sponge[16];
  uint32_t in_buf[8];
  uint32_t in_len;
  uint32_t out_buf[8];
  uint32_t out_len;
};
// First out-of-range access a guarded kernel skipped (count = accesses
// skipped since the last clear).  Tags name the kind of access.
struct GuardRecord {
  unsigned long long count, tag, offset, extent, block, thread, pad[2];
};
enum GuardTag : int {
  kGuardLoad = 1,       // LDE global load (offset / extent in words of the pass's input)
  kGuardStore = 2,      // LDE global store (offset / extent in words of the pass's output)
  kGuardRowRead = 10,   // row hashing: segment index / column
  kGuardTile = 100,     // LDE shared-memory tile index
  kGuardTwiddle = 101,  // LDE shared-memory twiddle index
  kGuardPowIndex = 102  // coset power-table exponent
};
// Asynchronous copy of a unit's record to host memory on st / synchronous clear.
cudaError_t lde_guard_fetch(GuardRecord* dst, cudaStream_t st);
cudaError_t lde_guard_clear();
cudaError_t hash_guard_fetch(GuardRecord* dst, cudaStream_t st);
cudaError_t hash_guard_clear();

// Per-field twiddle tables: lo[j] = w^j, hi[j] = w^(j * 2^14), w of order 2^S;
// `stage`: the per-stage tables of every sub-transform length 2^l, l = 1..12,
// in the layout the LDE kernels copy into shared memory (launch_stage_tables).
struct TwiddleTables {
  const uint32_t* lo;
  const uint32_t* hi;
  const uint32_t* stage;
};
constexpr uint32_t kTwiddleWords = 16384;     // words of lo, and of hi
constexpr uint32_t kStageTableWords = 32768;  // words of stage: 16380 two-word entries
// Fill `stage` (kStageTableWords words) from lo/hi of the same field.
cudaError_t launch_stage_tables(int field, TwiddleTables tw, uint32_t* stage, cudaStream_t st);
// Fold one codeword of 2^log_len EF4 elements to half length with the EF4
// challenge at beta (device, 4 words).
// With `inject` (2^(log_len-1) x 4 words) the folded row adds inject[r]: the
// reduced opening of the folded height (the commit-phase loop of
// TwoAdicFriPcs::open, mirrored by fri.rs:300-318).
cudaError_t launch_fri_fold_tw(int field, const uint32_t* cw, uint32_t log_len, const uint32_t* beta,
                               TwiddleTables tw, uint32_t* out, cudaStream_t st, const uint32_t* inject = nullptr);
// Fold (as launch_fri_fold_tw, with inject) and hash the folded codeword's
// leaves: leaves[k] = hash(out[2k] || out[2k+1]) (8 words), log_len >= 2.
cudaError_t launch_fri_fold_hash(int field, const uint32_t* cw, uint32_t log_len, const uint32_t* beta,
                                 TwiddleTables tw, uint32_t* out, const uint32_t* inject, uint32_t* leaves,
                                 cudaStream_t st);
// One shard of a codeword split by rows: cw holds the 4 n_leaves rows from
// row 2 row0 of a 2^log_len-row codeword; fold them (twiddles of their rows in
// the whole codeword) into out (2 n_leaves rows) and hash the leaves.
cudaError_t launch_fri_fold_hash_rows(int field, const uint32_t* cw, uint32_t log_len, uint64_t row0,
                                      uint64_t n_leaves, const uint32_t* beta, TwiddleTables tw, uint32_t* out,
                                      uint32_t* leaves, cudaStream_t st);
// Coefficients of the final polynomial (2^log_keep x 4 words) from the last
// codeword of 2^log_len EF4 elements; *err set if higher coefficients are nonzero.
cudaError_t launch_fri_final_poly(int field, const uint32_t* cw, uint32_t log_len, uint32_t log_keep,
                                  TwiddleTables tw, uint32_t* coeffs, uint32_t* err, cudaStream_t st);
// Observe an 8-element root, then sample 4 elements into beta_out (EF4).
cudaError_t launch_challenger_round(int field, DevChallenger* ch, const uint32_t* root, uint32_t* beta_out,
                                    cudaStream_t st);
// Levels above `level` (n_in <= 512 digests, a power of two) up to the root,
// written after it; with ch, then observe the root and sample beta_out (4 words).
cudaError_t launch_tree_top(int field, uint32_t* level, uint32_t n_in, DevChallenger* ch, uint32_t* beta_out,
                            cudaStream_t st);
// Observe n elements at vals.
cudaError_t launch_challenger_observe(int field, DevChallenger* ch, const uint32_t* vals, uint32_t n,
                                      cudaStream_t st);

// --- LDE kernels (ntt_kernels.cu) ----------------------------------------
// The committed LDE of one matrix is 2^b coset blocks of n rows (block cb =
// the evaluations on the coset shift * w_N^rev_b(cb) * H_n, bit-reversed).
// With shard_log = k > 0 (k <= b), only the 2^(b-k) blocks of shard s are
// computed, cb in [s * 2^(b-k), (s+1) * 2^(b-k)): rows [s N / 2^k, (s+1) N / 2^k)
// of the committed LDE; out, t2 and pw then hold those blocks only.
struct LdeMat {
  const uint32_t* in;  // n x w evaluations
  uint32_t* out;       // (n << (b - k)) x w, bit-reversed rows
  uint32_t* t1;        // n x w scratch (three-pass form only)
  uint32_t* t2;        // (n << (b - k)) x w scratch (three-pass form only)
  uint32_t* pw;        // 2^(b-k) tables of 8192 words: g_cb^i / n, two-level
  uint32_t log_n, log_b, w;
  uint32_t log_n1, log_n2; // three-pass split n = n1 * n2 (0 for the one-pass form)
  uint32_t shift;          // coset shift, Monty form
  uint32_t shard_log, shard;  // k and s above (0, 0: every block)
};
// Coset blocks an LDE computes (log2) and the first one.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint32_t lde_log_c(const LdeMat& m) { return m.log_b - m.shard_log; }
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint32_t lde_cb0(const LdeMat& m) { return m.shard << lde_log_c(m); }
constexpr int kLdeSmallMaxLog = 11;  // one-pass form handles n <= 2^11
constexpr uint32_t kLdeMaxLogN = 24;  // coset power tables cover exponents below 2^24
constexpr int kLdeBatch = 32;        // matrices per launch (descriptors travel as kernel parameters)
struct LdeBatch {
  uint32_t n;
  uint32_t pad;
  LdeMat m[kLdeBatch];
};
constexpr uint32_t kPwWords = 8192;  // words per (matrix, coset) power table
// Largest log_blowup an LDE accepts: the coset power tables of one matrix
// (kPwWords << log_blowup words) are indexed with 32-bit arithmetic.
constexpr uint32_t kLdeMaxLogBlowup = 16;

// Power tables then LDE kernels for `n` matrices (host descriptors, any
// count; launched in batches of kLdeBatch).  *launches counts kernels.
cudaError_t launch_lde(int field, const LdeMat* mats, uint32_t n, TwiddleTables tw, cudaStream_t st,
                       uint64_t* launches = nullptr);

// Choose the one-pass or three-pass form for one matrix (fills log_n1, log_n2).
// One-pass form for n <= 2^11; above, the four-step split n = n1 * n2 with
// log_n1 if it is a valid split (both factors 2^6 .. 2^12), else the default
// n1 = 2^ceil(log_n / 2).
void plan_lde_tiling(LdeMat& m, uint32_t log_n1 = 0);
bool lde_split_valid(uint32_t log_n, uint32_t log_n1);

}  // namespace pico
