/*
 * pico_gpu.h -- C ABI of the B200 trace-commitment path.
 *
 * The reference prover (brevis-network/pico) commits traces through Plonky3's
 * trait objects, selected by type aliases in its STARK configs:
 *   SC_Dft = Radix2DitParallel, SC_ValMmcs = MerkleTreeMmcs<..Poseidon2..>,
 *   SC_Pcs = TwoAdicFriPcs  (vm/src/configs/stark_config/kb_poseidon2.rs:15-27,
 *   bb_poseidon2.rs:15-27; PCS constructed at kb_poseidon2.rs:82-93).
 * A GPU-backed config swaps those aliases for Rust types whose methods call
 * the entry points below; the prover's call sites stay unchanged
 * (pcs.commit: vm/src/machine/prover.rs:102,244,415,540;
 *  get_evaluations_on_domain: prover.rs:469-489; pcs.open: prover.rs:589).
 *
 * Conventions
 *   - Field elements are u32 in Plonky3's Montgomery form (x * 2^32 mod p), the
 *     in-memory representation of KoalaBear / BabyBear (MontyField31), so Rust
 *     `Vec<KoalaBear>` buffers pass through without conversion.
 *   - Matrices are row-major, height = 2^log_height rows of `width` elements
 *     (RowMajorMatrix).
 *   - Every function returns a pico_status; nothing aborts, nothing throws
 *     across the boundary (precedent: the reference's own C ABI,
 *     gnark/field-ffi/src/koalabear.rs:6-21).  pico_gpu_last_error() returns a
 *     thread-local description of the last failure.
 *   - All functions are thread-safe; concurrent calls on one context overlap
 *     on the device (the reference commits chunks from rayon workers,
 *     vm/src/instances/machine/riscv.rs:234).
 */
#ifndef PICO_GPU_H
#define PICO_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PICO_GPU_ABI_VERSION 1u

typedef enum {
  PICO_OK = 0,
  PICO_ERR_INVALID_ARG = 1,
  PICO_ERR_OUT_OF_MEMORY = 2, /* device allocation failed or HBM budget exceeded */
  PICO_ERR_CUDA = 3,
  PICO_ERR_UNSUPPORTED = 4,
  PICO_ERR_TIMEOUT = 5,
  PICO_ERR_NOT_READY = 6, /* asynchronous request still in flight */
  PICO_ERR_CANCELLED = 7,
  PICO_ERR_NO_DEVICE = 8
} pico_status;

typedef enum { PICO_KOALABEAR = 0, PICO_BABYBEAR = 1 } pico_field;

/* Flags for commit / LDE / FRI calls. */
#define PICO_INPUT_DEVICE 0x1u /* input pointers are device pointers (else host) */
#define PICO_COMMIT_PLAIN 0x2u /* one matrix per launch (LDE and row hashing): the baseline form */
#define PICO_OUTPUT_DEVICE 0x4u /* output pointers are device pointers (else host) */
#define PICO_LDE_NATURAL_ORDER 0x8u /* coset_lde_batch: natural row order (Dft trait); default bit-reversed */
#define PICO_P2_FOUR_LANES 0x10u /* poseidon2_permute: four threads per state (shorter latency per state) */
#define PICO_QUOTIENT_CHUNKS 0x20u /* quotient_values: output split into its 2^log_quotient_degree chunks */

typedef struct pico_ctx pico_ctx;
/* Prover data of one commit: every LDE and every digest layer stays resident
 * on the device until pico_gpu_release (the Rust ProverData's Drop). */
typedef struct pico_commit pico_commit;
/* Resident layers of one FRI commit phase (codewords and their trees). */
typedef struct pico_fri pico_fri;
/* An asynchronous commit request (serving path). */
typedef struct pico_request pico_request;
/* One shard of a FRI commit phase split by rows over several devices. */
typedef struct pico_fri_shard pico_fri_shard;

typedef struct {
  const uint32_t *values; /* row-major 2^log_height x width, Monty form */
  uint32_t log_height;
  uint32_t width;
  uint32_t shift; /* LDE coset shift, Monty form: GENERATOR / domain.shift */
  uint32_t flags; /* PICO_MATRIX_* */
} pico_matrix;

/* pico_matrix.flags: the values are degree-4 extension elements (4 Monty words
 * each, c0..c3) and `width` counts them.  The matrix is committed as the base
 * matrix of 4 * width columns that flatten_to_base makes of it (the
 * permutation traces, vm/src/machine/prover.rs:404-415) -- the same words, so
 * nothing is copied or rearranged. */
#define PICO_MATRIX_EXT4 0x1u

typedef struct {
  uint64_t hbm_budget_bytes; /* admission budget; 0 = 90% of free HBM at init */
  uint32_t n_streams;        /* device streams for concurrent requests; 0 = 8 */
  uint32_t flags;
  uint32_t max_inflight;     /* serving: requests on the device at once; 0 = n_streams */
  uint32_t max_group;        /* serving: queued requests admitted together as one group that shares its
                                LDE and row-hashing launches (batched device-input requests of one field);
                                0 = 8, 1 = each request alone, at most 16 */
  uint32_t reserved[4];
} pico_config;

/* Device-side timing and work counts of one commit, from CUDA events recorded
 * on the commit's stream (milliseconds). */
typedef struct {
  double total_ms;   /* first input copy or launch -> root ready */
  double h2d_ms;     /* host -> device input copies (host inputs only) */
  double lde_ms;     /* coset LDE kernels, all matrices */
  double leaves_ms;  /* leaf hashing of the tallest height group */
  double tree_ms;    /* compression levels, including injected rows */
  uint64_t cells;    /* trace cells before blowup */
  uint64_t lde_cells;
  uint64_t permutations; /* Poseidon2 permutations in the tree */
  uint64_t leaf_permutations;
  uint64_t lde_bytes; /* algorithmic LDE bytes: 4 * (cells + lde_cells) */
  uint64_t launches;  /* kernels this library launched for the commit */
} pico_commit_stats;

/* Duplex challenger state, DuplexChallenger<F, Perm, 16, 8> (Monty form). */
typedef struct {
  uint32_t sponge[16];
  uint32_t in_buf[8];
  uint32_t in_len;
  uint32_t out_buf[8];
  uint32_t out_len;
} pico_challenger;

/* ---- DuplexChallenger on the host --------------------------------------
 * observe / sample of DuplexChallenger<F, Perm, 16, 8>
 * (vm/src/compiler/recursion/circuit/challenger.rs:89-106 observe and sample,
 * 223-234 duplexing), the transcript steps pico_gpu_pcs_open runs on the host,
 * with the same Poseidon2-16.  observe absorbs n field elements (Monty form)
 * one at a time; sample writes the next n samples (Monty form).  No device is
 * needed.  The host permutation uses AVX-512 or AVX2 when the CPU has them;
 * the environment variable PICO_HOST_SIMD (0 scalar, 2 at most AVX2) caps it. */
pico_status pico_gpu_challenger_observe(pico_field field, pico_challenger *ch, const uint32_t *values, uint64_t n);
pico_status pico_gpu_challenger_sample(pico_field field, pico_challenger *ch, uint32_t *out, uint64_t n);

/* ---- context ------------------------------------------------------------ */
pico_status pico_gpu_init(int device, const pico_config *cfg, pico_ctx **out);
pico_status pico_gpu_shutdown(pico_ctx *ctx);
const char *pico_gpu_last_error(void);
uint32_t pico_gpu_abi_version(void);
/* Bytes currently reserved by resident commits / in-flight requests, and the budget. */
pico_status pico_gpu_memory(pico_ctx *ctx, uint64_t *reserved, uint64_t *budget);
/* Grow the device's stream-ordered memory pool, which every device buffer of
 * this library comes from, to hold at least `bytes` (at most the context's
 * budget) by allocating and freeing that much once, so that later commits and
 * served requests take memory from the pool instead of growing it: growth is
 * synchronous, and the first group of served requests that needed more than
 * the pool held stalled for up to 0.3 s in measurement.  The pool keeps its
 * memory until the process exits (other allocators of the process cannot use
 * it).  pool_bytes (nullable) receives what the pool then holds. */
pico_status pico_gpu_reserve_pool(pico_ctx *ctx, uint64_t bytes, uint64_t *pool_bytes);
/* Device bytes a commit of these matrices would reserve against the budget
 * (pico_gpu_commit / pico_gpu_submit_commit with the same arguments):
 * `resident` stays reserved until the commit is released (LDEs, digest
 * layers), `scratch` only while it runs.  Validates the descriptors exactly as
 * those calls do; needs no device.  No counterpart in the reference (its CPU
 * commit has no admission step); a serving front end sizes requests with it. */
pico_status pico_gpu_commit_bytes(pico_field field, const pico_matrix *mats, uint32_t n_mats, uint32_t log_blowup,
                                  uint32_t flags, uint64_t *resident, uint64_t *scratch);

/* ---- Pcs::commit ---------------------------------------------------------
 * TwoAdicFriPcs::commit (Plonky3 @ brevis-network/Plonky3 f5056c9, called at
 * vm/src/machine/prover.rs:102,244,415,540): per matrix a coset LDE with
 * log_blowup and the matrix's shift, rows bit-reversed, then one
 * MerkleTreeMmcs commit over all LDEs (stable sort by height, rows of shorter
 * matrices injected at their level).  Heights must be powers of two.
 * `out` (nullable) receives the resident prover data; root receives the
 * 8-element commitment (host memory). */
pico_status pico_gpu_commit(pico_ctx *ctx, pico_field field, const pico_matrix *mats, uint32_t n_mats,
                            uint32_t log_blowup, uint32_t flags, pico_commit **out, uint32_t root[8]);
pico_status pico_gpu_release(pico_ctx *ctx, pico_commit *c);
/* Timing of a finished commit (waits for it), and of the last synchronous
 * commit made by the calling thread (also when its prover data was not kept). */
pico_status pico_gpu_commit_stats(const pico_commit *c, pico_commit_stats *out);
pico_status pico_gpu_last_commit_stats(pico_commit_stats *out);

/* Pcs::get_evaluations_on_domain / open_batch row reads (prover.rs:469-489):
 * rows [row_begin, row_end) of committed LDE `mat_idx` (input order), in the
 * committed (bit-reversed) row order.  Output is host memory unless
 * PICO_OUTPUT_DEVICE. */
pico_status pico_gpu_lde_rows(pico_ctx *ctx, const pico_commit *c, uint32_t mat_idx, uint64_t row_begin,
                              uint64_t row_end, uint32_t *out, uint32_t flags);
/* Pcs::get_evaluations_on_domain for the domain g * H_(2^log_domain), no taller
 * than the committed LDE (the quotient-domain reads of compute_quotient_values,
 * vm/src/machine/prover.rs:469-489): the first 2^log_domain committed rows,
 * returned in natural order (row k = evaluation at g * w^k), row-major
 * 2^log_domain x width words; host memory unless PICO_OUTPUT_DEVICE. */
pico_status pico_gpu_evaluations_on_domain(pico_ctx *ctx, const pico_commit *c, uint32_t mat_idx,
                                           uint32_t log_domain, uint32_t *out, uint32_t flags);
/* Shape of a committed LDE: log2 height and width. */
pico_status pico_gpu_lde_shape(const pico_commit *c, uint32_t mat_idx, uint32_t *log_height, uint32_t *width);
/* Digest layer `level` (0 = leaves) of the commit's tree: 2^(log_max - level)
 * digests of 8 words. */
pico_status pico_gpu_digest_layer(pico_ctx *ctx, const pico_commit *c, uint32_t level, uint32_t *out,
                                  uint32_t flags);
/* Mmcs::open_batch: the opened rows of every matrix at `index` (an index into
 * the tallest LDE; shorter matrices use index >> (log_max - log_h)) and the
 * sibling path.  rows_out receives the concatenated rows in input order
 * (sum of widths words); path_out receives log_max digests of 8 words. */
pico_status pico_gpu_open_batch(pico_ctx *ctx, const pico_commit *c, uint64_t index, uint32_t *rows_out,
                                uint32_t *path_out);

/* ---- Dft / Mmcs / permutation granularity -------------------------------- */
/* Radix2DitParallel::coset_lde_batch (SC_Dft, kb_poseidon2.rs:25): n x w
 * evaluations on the two-adic subgroup -> 2^log_blowup * n evaluations on
 * shift * H, bit-reversed rows unless PICO_LDE_NATURAL_ORDER. */
pico_status pico_gpu_coset_lde_batch(pico_ctx *ctx, pico_field field, const uint32_t *in, uint32_t log_n,
                                     uint32_t width, uint32_t log_blowup, uint32_t shift, uint32_t *out,
                                     uint32_t flags);
/* Allocation-free variant of pico_gpu_coset_lde_batch.  No counterpart in the
 * reference: it exists for callers that cannot let this library allocate
 * device memory (a prover that has reserved all of HBM for its own arena, or
 * a latency-bound loop that cannot afford cudaMalloc/cudaFree's device-wide
 * synchronisation).  `in` and `out` are device buffers owned by the caller;
 * scratch comes from a 32 MiB array declared in device memory by the library
 * (held by every GPU that loads it until exit), so LDEs needing more than
 * 2^b*8192 + n*w*(1 + 2^b) > 8 Mi words of scratch are rejected with
 * PICO_ERR_INVALID_ARG.  No context is needed; work is enqueued on `stream`
 * (a cudaStream_t, 0 = legacy default) and is complete when the stream
 * reaches that point.  All calls share the scratch array: calls that overlap
 * on the GPU race and must be serialised.  The first call on a device does a
 * one-time set-up (symbol lookup, twiddle fill, synchronise) and should come
 * before any stream capture. */
pico_status pico_gpu_coset_lde_batch_noalloc(pico_field field, const uint32_t *in, uint32_t log_n, uint32_t width,
                                             uint32_t log_blowup, uint32_t shift, uint32_t *out, void *stream);
/* Completion check of pico_gpu_coset_lde_batch_noalloc calls: waits for
 * `stream`, then reports whether any LDE kernel skipped an out-of-range access
 * since the last check (PICO_ERR_CUDA with the first such access in
 * pico_gpu_last_error; the result of that call is then wrong) and clears the
 * record.  Allocates nothing.  The record is per device and shared with the
 * context-based LDE and commit calls, which report and clear it themselves. */
pico_status pico_gpu_noalloc_status(void *stream);
/* MerkleTreeMmcs::commit (SC_ValMmcs, kb_poseidon2.rs:19-20) over matrices
 * that are already extended: mats[i].log_height is the matrix's own height,
 * shift is ignored. */
pico_status pico_gpu_mmcs_commit(pico_ctx *ctx, pico_field field, const pico_matrix *mats, uint32_t n_mats,
                                 uint32_t flags, pico_commit **out, uint32_t root[8]);
/* One shard of TwoAdicFriPcs::commit (prover.rs:102) split by rows over
 * 2^log_shards devices (no counterpart in the reference, which commits on one
 * host).  Shard s holds rows [s N / 2^k, (s + 1) N / 2^k) of every committed
 * LDE (N its height, k = log_shards), i.e. the LDE's coset blocks
 * s 2^(b-k) .. (s + 1) 2^(b-k) - 1: each shard computes them from the whole
 * trace, with no exchange between devices, so k <= log_blowup.  It also builds
 * the Merkle tree over its rows (rows of shorter matrices injected where
 * their heights meet, as in the full tree); that tree is the full tree's
 * subtree under the node at depth k, index s, and `root` receives it.
 * pico_gpu_merkle_top turns the 2^k shard roots into the commitment root.  The
 * prover data holds the shard's rows (lde_rows, digest_layer and open_batch
 * count them from the shard's first row); the calls that need every committed
 * row (pcs_open, open_values, reduced_opening, evaluations_on_domain,
 * quotient_values) refuse it with PICO_ERR_UNSUPPORTED. */
pico_status pico_gpu_commit_shard(pico_ctx *ctx, pico_field field, const pico_matrix *mats, uint32_t n_mats,
                                  uint32_t log_blowup, uint32_t log_shards, uint32_t shard, uint32_t flags,
                                  pico_commit **out, uint32_t root[8]);
/* The top log_shards levels of a Merkle tree on the host: the 2^log_shards
 * shard roots (8 words each, in shard order) compressed pairwise up to the
 * root (MerkleTreeMmcs compression; no device needed). */
pico_status pico_gpu_merkle_top(pico_field field, const uint32_t *roots, uint32_t log_shards, uint32_t root[8]);
/* The last log_shards digests of a Merkle path through shard `shard` of a
 * row-split commit (lowest level first): pico_gpu_open_batch on the shard's
 * prover data, at the index's row within the shard, gives the opened rows and
 * the path up to the shard's root; these siblings complete the path of the
 * whole commit (Mmcs::open_batch, checked as fri.rs:389-436 checks it). */
pico_status pico_gpu_merkle_top_path(pico_field field, const uint32_t *roots, uint32_t log_shards, uint32_t shard,
                                     uint32_t *path);
/* Poseidon2KoalaBear<16> / Poseidon2BabyBear<16> on n states of 16 words, in place. */
pico_status pico_gpu_poseidon2_permute(pico_ctx *ctx, pico_field field, uint32_t *states, uint64_t n,
                                       uint32_t flags);

/* ---- FRI commit phase (inside TwoAdicFriPcs::open, prover.rs:589) ----------
 * codeword: 2^log_n degree-4 extension elements (4 words each, c0..c3), in
 * bit-reversed evaluation order.  Rounds: commit the codeword as a
 * (len/2) x 2 extension matrix flattened to 8 base columns (ExtensionMmcs),
 * observe the root, sample beta (sample_ext), fold with arity 2; stop at
 * length 2^(log_blowup + log_final_len).  If betas_in is non-null the round
 * challenges are taken from it (rounds x 4 words) instead of the challenger.
 * ch (in/out, used when betas_in is null) is the prover's challenger state.
 * Outputs (host): roots (rounds x 8), betas (rounds x 4), final_out
 * (2^log_final_len x 4: with log_final_len = 0 the single final_poly element).
 * `out` (nullable) keeps every codeword and tree resident for queries. */
pico_status pico_gpu_fri_commit_phase(pico_ctx *ctx, pico_field field, const uint32_t *codeword, uint32_t log_n,
                                      uint32_t log_blowup, uint32_t log_final_len, const uint32_t *betas_in,
                                      pico_challenger *ch, uint32_t flags, uint32_t *roots, uint32_t *betas,
                                      uint32_t *final_out, uint32_t *n_rounds, pico_fri **out);
pico_status pico_gpu_fri_release(pico_ctx *ctx, pico_fri *f);
/* Codeword of round r (r = 0 is the input) as 2^(log_n - r) x 4 words. */
pico_status pico_gpu_fri_layer(pico_ctx *ctx, const pico_fri *f, uint32_t round, uint32_t *out, uint32_t flags);

/* The commit phase of a codeword split by rows over 2^k devices (no
 * counterpart in the reference, which runs it on one host).  Shard s holds
 * rows [s N / 2^k, (s + 1) N / 2^k) of the N-row EF4 codeword (committed
 * order, 4 words per row), the row partition of pico_gpu_commit_shard.  A
 * round's tree hashes rows 2i, 2i + 1 into leaf i, so a shard's rows make the
 * subtree under node s at depth k, and the fold pairs the same rows, so the
 * next round's shard rows come from this shard's alone.  Per round the caller
 * gathers the 2^k shard roots (pico_gpu_merkle_top gives the round's root),
 * observes it and samples beta on its challenger, and calls fold with beta;
 * when the shards are short it gathers the codeword (pico_gpu_fri_shard_rows)
 * and finishes with pico_gpu_fri_commit_phase on one device, continuing the
 * same challenger.  begin: the shard's rows (host, or device with
 * PICO_INPUT_DEVICE) of a 2^log_n-row codeword, and its round-0 subtree root.
 * fold: the next round's rows and subtree root (needs at least 4 rows). */
pico_status pico_gpu_fri_shard_begin(pico_ctx *ctx, pico_field field, const uint32_t *rows, uint32_t log_n,
                                     uint32_t log_shards, uint32_t shard, uint32_t flags, pico_fri_shard **out,
                                     uint32_t root[8]);
pico_status pico_gpu_fri_shard_fold(pico_fri_shard *fs, const uint32_t beta[4], uint32_t root[8]);
pico_status pico_gpu_fri_shard_rows(pico_fri_shard *fs, uint32_t *out, uint32_t flags);
pico_status pico_gpu_fri_shard_release(pico_fri_shard *fs);

/* ---- PCS opening (TwoAdicFriPcs::open, vm/src/machine/prover.rs:589) -------
 * Every step follows the Pico verifier (vm/src/compiler/recursion/circuit/
 * fri.rs:77-436): opened values p(z) by barycentric evaluation over each
 * matrix's low coset; all of them observed (4 coefficients each, batch /
 * matrix / point / column order), then alpha sampled; one reduced opening
 * per LDE height; the FRI commit phase folds the tallest one and adds each
 * shorter one at its height; the final element is observed, a proof-of-work
 * witness found (the smallest that passes), and the query indices sampled.
 *
 * One batch: a resident commitment (committed with the same log_blowup) and,
 * for each of its matrices in commit input order, the points it is opened at
 * (degree-4 extension elements, 4 Monty words each, concatenated in matrix
 * order; n_points[m] may be 0). */
typedef struct {
  const pico_commit *commit;
  const uint32_t *n_points;
  const uint32_t *points;
} pico_open_batch;

typedef struct {
  uint32_t log_blowup;
  uint32_t num_queries;
  uint32_t proof_of_work_bits; /* at most 24 */
  uint32_t reserved;
} pico_fri_params;

typedef struct {
  float ms_values;  /* device: inverse denominators and opened values */
  float ms_reduce;  /* device: reduced openings */
  float ms_fri;     /* device: commit phase */
  float ms_grind;   /* device: proof of work */
  float ms_queries; /* device: query records */
  float ms_total;   /* wall clock of the call */
  uint64_t value_cells;  /* low-coset cells read per opened point */
  uint64_t reduce_cells; /* committed cells read by the reduction */
  uint32_t launches;
  uint32_t rounds;
} pico_open_stats;

/* Output sizes: opened-value words (sum of n_points x width x 4), FRI rounds
 * (log of the tallest LDE height - log_blowup) and words per query record. */
pico_status pico_gpu_open_sizes(const pico_open_batch *batches, uint32_t n_batches, uint32_t log_blowup,
                                uint64_t *value_words, uint32_t *rounds, uint64_t *query_words);

/* The whole opening.  ch: the prover's challenger (in/out).  Outputs (host):
 * values (value_words), commit_roots (rounds x 8), betas (rounds x 4,
 * nullable), final_poly (4), pow_witness (1, Monty), query_indices
 * (num_queries), queries (num_queries x query_words): per query, for each
 * batch the opened row of every matrix (input order) then the batch's Merkle
 * path (leaf level first); then for each FRI round the sibling value (4
 * words) and the path in that round's tree.  stats nullable. */
pico_status pico_gpu_pcs_open(pico_ctx *ctx, const pico_open_batch *batches, uint32_t n_batches,
                              const pico_fri_params *params, pico_challenger *ch, uint32_t *values,
                              uint32_t *commit_roots, uint32_t *betas, uint32_t final_poly[4], uint32_t *pow_witness,
                              uint32_t *query_indices, uint32_t *queries, pico_open_stats *stats);

/* The first step alone: opened values (value_words), no transcript. */
pico_status pico_gpu_open_values(pico_ctx *ctx, const pico_open_batch *batches, uint32_t n_batches,
                                 uint32_t log_blowup, uint32_t *values);

/* The reduced opening of LDE height 2^log_height (2^log_height x 4 words) for
 * the given opened values and alpha, as fed to the commit phase.  It is formed
 * on the low coset and extended (it is a polynomial of degree < n there), which
 * is the reference's row-by-row value when `values` are the opened values
 * pico_gpu_open_values returns.  A point on a committed coset is rejected
 * (PICO_ERR_INVALID_ARG) by all three opening calls. */
pico_status pico_gpu_reduced_opening(pico_ctx *ctx, const pico_open_batch *batches, uint32_t n_batches,
                                     uint32_t log_blowup, const uint32_t *values, const uint32_t alpha[4],
                                     uint32_t log_height, uint32_t *out);

/* ---- quotient values (compute_quotient_values, vm/src/machine/utils.rs:201-350,
 * called from vm/src/machine/prover.rs:457-511) ---------------------------------
 * A chip's quotient over its quotient domain GENERATOR * <w_Q>,
 * Q = 2^(log_trace_height + log_quotient_degree), in natural order: for each
 * point x the chip's constraints are folded as the prover's
 * ProverConstraintFolder folds them (every assertion: acc = acc * alpha + c,
 * vm/src/machine/folder.rs:223-227,321-327) over the local row and the next
 * row (x * w_n), and the value is acc / Z_H(x), with the Lagrange selectors
 * of vm/src/compiler/recursion/circuit/domain.rs:48-66.
 *
 * The traces are read from resident commits (no copy): main is required,
 * preprocessed and permutation are optional (commit NULL); each must have
 * been committed with the standard LDE shift and at least Q rows.  The
 * permutation trace is its base flattening (4 words per extension column,
 * as PICO_MATRIX_EXT4 commits it).
 *
 * The constraints are a straight-line program over 64 base and 16 extension
 * registers, what a Rust shim emits from the chip's symbolic constraints
 * (Plonky3 SymbolicExpression): op, dst, a, b per instruction.  For the loads
 * b = 1 reads the next row.  Constants are Monty form.  public_values (n_public
 * words), perm_challenges (n_challenges x 4), regional_sum (4, nullable),
 * global_sum (14 coordinates of the septic digest, nullable), alpha (4).
 * out: Q x 4 words, host memory unless PICO_OUTPUT_DEVICE.  With
 * PICO_QUOTIENT_CHUNKS the output is the D = 2^log_quotient_degree chunks
 * that the prover commits next (prover.rs:517-538: flatten_to_base, then the
 * domain's split_evals and split_domains): chunk j, n = 2^log_trace_height
 * EF4 values at out + 4 n j, holds the points i = j, j + D, j + 2D, ..., the
 * evaluations on GENERATOR * w_Q^j * <w_n>, so each chunk commits as a
 * PICO_MATRIX_EXT4 matrix of height n and LDE shift w_Q^-j.  No counterpart in
 * the reference's types for the program itself: the reference evaluates the
 * Rust `eval` directly. */
typedef enum {
  PICO_Q_MAIN = 1,        /* base[dst] = main column a (b: next row) */
  PICO_Q_PREP = 2,        /* base[dst] = preprocessed column a */
  PICO_Q_PERM = 3,        /* ext[dst] = permutation extension column a */
  PICO_Q_CONST = 4,       /* base[dst] = a (Monty form) */
  PICO_Q_PUBLIC = 5,      /* base[dst] = public_values[a] */
  PICO_Q_FIRST = 6,       /* base[dst] = is_first_row */
  PICO_Q_LAST = 7,        /* base[dst] = is_last_row */
  PICO_Q_TRANSITION = 8,  /* base[dst] = is_transition */
  PICO_Q_ADD = 9,         /* base[dst] = base[a] + base[b]; SUB, MUL alike */
  PICO_Q_SUB = 10,
  PICO_Q_MUL = 11,
  PICO_Q_EADD = 12,       /* ext[dst] = ext[a] + ext[b]; ESUB, EMUL alike */
  PICO_Q_ESUB = 13,
  PICO_Q_EMUL = 14,
  PICO_Q_EMB = 15,        /* ext[dst] = base[a] */
  PICO_Q_EMULB = 16,      /* ext[dst] = ext[a] * base[b] */
  PICO_Q_CHALLENGE = 17,  /* ext[dst] = perm_challenges[a] */
  PICO_Q_REGIONAL = 18,   /* ext[dst] = regional cumulative sum */
  PICO_Q_GLOBAL = 19,     /* base[dst] = global cumulative sum coordinate a */
  PICO_Q_ASSERT = 20,     /* acc = acc * alpha + base[a] */
  PICO_Q_EASSERT = 21     /* acc = acc * alpha + ext[a] */
} pico_constraint_opcode;

typedef struct {
  uint32_t op, dst, a, b;
} pico_constraint_op;

typedef struct {
  const pico_commit *commit; /* NULL: the trace is absent */
  uint32_t mat_idx;          /* matrix of the commit (input order) */
  uint32_t reserved;
} pico_trace_ref;

pico_status pico_gpu_quotient_values(pico_ctx *ctx, pico_trace_ref preprocessed, pico_trace_ref main,
                                     pico_trace_ref permutation, uint32_t log_trace_height,
                                     uint32_t log_quotient_degree, const pico_constraint_op *program,
                                     uint32_t n_ops, const uint32_t *public_values, uint32_t n_public,
                                     const uint32_t *perm_challenges, uint32_t n_challenges,
                                     const uint32_t regional_sum[4], const uint32_t global_sum[14],
                                     const uint32_t alpha[4], uint32_t *out, uint32_t flags);

/* ---- serving: asynchronous commits ----------------------------------------
 * pico_gpu_submit_commit copies the host matrices it is given before it
 * returns (the caller may reuse them) and queues the commit.  A request is
 * admitted to the device when the HBM budget has room for its LDEs, digest
 * layers and scratch; admitted requests run concurrently on separate streams.
 * pico_gpu_wait blocks up to timeout_ms (< 0: forever) for completion and then
 * hands over the prover data and root exactly as pico_gpu_commit would. */
pico_status pico_gpu_submit_commit(pico_ctx *ctx, pico_field field, const pico_matrix *mats, uint32_t n_mats,
                                   uint32_t log_blowup, uint32_t flags, pico_request **out);
pico_status pico_gpu_poll(pico_ctx *ctx, pico_request *req);
pico_status pico_gpu_wait(pico_ctx *ctx, pico_request *req, int64_t timeout_ms, pico_commit **out,
                          uint32_t root[8]);
/* Cancel a request that has not been admitted yet; admitted requests finish. */
pico_status pico_gpu_cancel(pico_ctx *ctx, pico_request *req);
/* Timing of a finished request: queue wait and device time in microseconds. */
pico_status pico_gpu_request_times(const pico_request *req, double *queued_us, double *run_us);
pico_status pico_gpu_request_free(pico_ctx *ctx, pico_request *req);

/* ---- autotuning (no counterpart in the reference; Plonky3's CPU path has
 * nothing to tune) -----------------------------------------------------------
 * pico_gpu_autotune times, on this device, the candidate four-step splits
 * n = n1 * n2 of the coset LDE for every height 2^log_n_min .. 2^log_n_max
 * that uses the three-pass form (n > 2^11), and the row-hashing block size,
 * and keeps the fastest in the context; later commits and LDEs of that field
 * use them.  Results are bit-identical for every choice.  ms_out (nullable)
 * receives 3 times per height (splits ceil(log_n/2) - 1, + 0, + 1; 0 where a
 * split is not valid) followed by 3 times for blocks 64, 128, 256.  Call it
 * before submitting work that should use the tuned values. */
pico_status pico_gpu_autotune(pico_ctx *ctx, pico_field field, uint32_t log_n_min, uint32_t log_n_max,
                              float *ms_out);
/* Read (and if set_log_n1 != 0, first set) the split used at height 2^log_n:
 * *log_n1_out = log2 n1, or 0 for the one-pass form. */
pico_status pico_gpu_lde_split(pico_ctx *ctx, pico_field field, uint32_t log_n, uint32_t set_log_n1,
                               uint32_t *log_n1_out);

/* ---- test hook (no counterpart in the reference) ----------------------------
 * Failure injection on the host: after `after` more device allocations made by
 * this library (any context, any thread), the next one fails as if the device
 * were out of memory (PICO_ERR_OUT_OF_MEMORY), then injection switches off;
 * after < 0 switches it off.  Tests use it to check that a failed commit
 * returns its budget and buffers and leaves the context usable. */
pico_status pico_gpu_test_fail_allocations(int64_t after);

#ifdef __cplusplus
}
#endif
#endif /* PICO_GPU_H */
