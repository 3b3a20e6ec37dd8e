/*
 * CPU oracle for the trace-commitment path: test infrastructure only.
 *
 * A plain-C restatement of the reference's hot-path arithmetic (Plonky3 as
 * pinned by brevis-network/pico, restated from the Pico-owned files cited in
 * oracle.c).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker or the timed CPU baseline; the
 * product library never links it.
 *
 * All buffers at this interface hold field elements in Plonky3's Montgomery
 * form (x * 2^32 mod p, the MontyField31 storage), exactly as the prover hands
 * them over.  Internally the oracle computes in canonical form with plain
 * 64-bit remainder arithmetic, so it shares no reduction tricks with the GPU.
 *
 * Parity status: the Poseidon2 permutation is pinned by the reference's
 * known-answer tests (gnark/poseidon2/poseidon2_{koalabear,babybear}_test.go).
 * Sponge, compression, mixed-height MMCS, FRI fold and challenger follow the
 * reference's verifier restatements.  The two-adic generators are derived
 * (GENERATOR^((p-1)/2^S)); no reference file pins them.
 */
#ifndef PICO_ORACLE_H
#define PICO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_KOALABEAR = 0, ORC_BABYBEAR = 1 };

/* Return codes. */
enum { ORC_OK = 0, ORC_EINVAL = 1, ORC_ENOMEM = 2 };

/* Duplex challenger state (Monty form), DuplexChallenger<F, Perm, 16, 8>. */
typedef struct {
    uint32_t sponge[16];
    uint32_t in_buf[8];
    uint32_t in_len;
    uint32_t out_buf[8];
    uint32_t out_len;
} orc_challenger;

uint32_t orc_prime(int field);
uint32_t orc_to_monty(int field, uint32_t x);
uint32_t orc_from_monty(int field, uint32_t x);
/* two_adic_generator(bits) in canonical form. */
uint32_t orc_two_adic_generator(int field, uint32_t bits);
uint32_t orc_generator(int field);
int orc_num_threads(void);
void orc_set_threads(int n);
/* The synthetic-input stream of the benchmarks, in Monty form: output i is the
 * i-th SplitMix64 draw (state seed + k * 0x9E3779B97F4A7C15, k = 1, 2, ...)
 * shifted right by 33 whose value is below p; draws >= p are skipped.  The
 * same stream as pico_b200.fields.uniform, for inputs too large for numpy. */
void orc_uniform_monty(int field, uint64_t seed, uint64_t n, uint32_t *out);

/* In-place Poseidon2-16 on n states (Monty form). */
int orc_permute(int field, uint32_t *states, size_t n);
/* In-place Poseidon2-16 on one state in canonical form (for KATs). */
int orc_permute_canonical(int field, uint32_t state[16]);

/* PaddingFreeSponge<16,8,8> over `len` Monty elements -> 8-element digest. */
int orc_hash(int field, const uint32_t *in, size_t len, uint32_t out[8]);
/* TruncatedPermutation<2,8,16>: permute(left || right)[0..8]. */
int orc_compress(int field, const uint32_t left[8], const uint32_t right[8], uint32_t out[8]);

/*
 * MerkleTreeMmcs::commit over matrices of power-of-two heights (row-major,
 * Monty).  `layers` (nullable) receives every digest layer from the leaves up
 * to the root, concatenated: (2*H_max - 1) * 8 words.
 */
int orc_mmcs_commit(int field, uint32_t n_mats, const uint32_t *const *mats,
                    const uint64_t *heights, const uint32_t *widths,
                    uint32_t root[8], uint32_t *layers);

/*
 * Radix2DitParallel::coset_lde_batch: n = 2^log_n evaluations on the two-adic
 * subgroup (row-major n x w) -> evaluations on shift * H_{n*2^b}.  If
 * bitrev_rows is nonzero the rows are bit-reversed as TwoAdicFriPcs::commit
 * does before hashing.
 */
int orc_coset_lde(int field, const uint32_t *in, uint32_t log_n, uint32_t w,
                  uint32_t log_blowup, uint32_t shift_monty, int bitrev_rows,
                  uint32_t *out);

/*
 * TwoAdicFriPcs::commit: per matrix coset LDE with shift = GENERATOR /
 * domain_shift (passed precomputed in `shifts`, Monty), bit-reversed rows,
 * then one MMCS commit over all.  `ldes` (nullable array of n_mats pointers)
 * receives each LDE; `layers` as in orc_mmcs_commit.
 */
int orc_pcs_commit(int field, uint32_t n_mats, const uint32_t *const *mats,
                   const uint32_t *log_heights, const uint32_t *widths,
                   const uint32_t *shifts, uint32_t log_blowup,
                   uint32_t root[8], uint32_t *const *ldes, uint32_t *layers);

void orc_challenger_init(orc_challenger *ch);
void orc_challenger_observe(int field, orc_challenger *ch, uint32_t v);
uint32_t orc_challenger_sample(int field, orc_challenger *ch);

/*
 * FRI commit phase on one degree-4 extension codeword (N = 2^log_n rows of 4
 * Monty words, bit-reversed evaluation order).  Folds with arity 2 until the
 * length is 2^(log_blowup + log_final_len).  Per round: commit the codeword as
 * an (N/2) x 2 extension matrix (flattened to 8 base columns), observe the
 * root, sample beta (or take betas_in[round] if betas_in is non-null), fold.
 * With log_final_len == 0 the result is Plonky3's single final_poly element
 * (observed into the challenger); otherwise the 2^log_final_len coefficients.
 * Outputs: roots (rounds x 8), betas (rounds x 4), final_out (2^log_final_len
 * x 4, coefficients).  Returns the number of rounds via *rounds_out.
 */
int orc_fri_commit_phase(int field, const uint32_t *codeword, uint32_t log_n,
                         uint32_t log_blowup, uint32_t log_final_len,
                         const uint32_t *betas_in, orc_challenger *ch,
                         uint32_t *roots, uint32_t *betas, uint32_t *final_out,
                         uint32_t *rounds_out);

/* Extension-field helpers (Monty in/out), for tests. */
void orc_ext_mul(int field, const uint32_t a[4], const uint32_t b[4], uint32_t out[4]);
void orc_ext_inv(int field, const uint32_t a[4], uint32_t out[4]);

/*
 * One batch of TwoAdicFriPcs::open: a committed batch and, per matrix, the
 * points it is opened at.  Prover fields: ldes (bit-reversed LDE rows, Monty)
 * and layers (the batch's digest layers as orc_mmcs_commit writes them).
 * Verifier field: root.  Points are degree-4 extension elements (4 Monty
 * words each), concatenated in matrix order.
 */
typedef struct {
    uint32_t n_mats;
    const uint32_t *const *ldes;
    const uint32_t *log_heights; /* log2 of the LDE heights */
    const uint32_t *widths;
    const uint32_t *n_points;
    const uint32_t *points;
    const uint32_t *layers;
    const uint32_t *root;
} orc_open_batch;

/* Opened values p_m(z) of one batch, ordered matrix, point, column (4 words each). */
int orc_open_values(int field, const orc_open_batch *b, uint32_t log_blowup, uint32_t *values);
/* The reduced opening of LDE height 2^log_height (2^log_height x 4 words). */
int orc_reduce_openings(int field, const orc_open_batch *batches, uint32_t n_batches, const uint32_t *values,
                        const uint32_t alpha[4], uint32_t log_height, uint32_t *ro_out);
/* Words of one query record (see orc_pcs_open). */
uint64_t orc_open_query_words(const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup);
/*
 * TwoAdicFriPcs::open: opened values, alpha, reduced openings, FRI commit phase
 * with the shorter reduced openings added at their heights, proof-of-work
 * witness (the smallest that passes), query indices and query records.
 * A query record holds, for each batch, the opened row of every matrix (input
 * order) and the batch's Merkle path (leaf level first); then, for each FRI
 * round, the sibling value (4 words) and the path in that round's tree.
 */
int orc_pcs_open(int field, const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup,
                 uint32_t num_queries, uint32_t pow_bits, orc_challenger *ch, uint32_t *values,
                 uint32_t *roots, uint32_t *betas, uint32_t final_poly[4], uint32_t *pow_witness,
                 uint32_t *indices, uint32_t *queries, uint32_t *rounds_out);
/* The Pico verifier's checks on an opening proof; 0 when it verifies, else
 * the failing check (10 proof of work, 11 input batch path, 12 reduced
 * opening at the blowup height, 13 commit-phase path, 14 final polynomial). */
int orc_verify_open(int field, const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup,
                    uint32_t num_queries, uint32_t pow_bits, orc_challenger *ch, const uint32_t *values,
                    const uint32_t *roots, uint32_t n_rounds, const uint32_t final_poly[4], uint32_t pow_witness,
                    const uint32_t *queries, uint32_t *indices_out);

/* ---- compute_quotient_values (vm/src/machine/utils.rs:201-350) ----------
 * A chip's constraints as a register program (the same op list the GPU entry
 * point pico_gpu_quotient_values takes): op, dst, a, b per instruction, base
 * registers (< 64) and extension registers (< 16).  Folded as the prover's
 * ProverConstraintFolder does (vm/src/machine/folder.rs:223-227,321-327):
 * each assertion does acc = acc * alpha + x; the quotient at a point is
 * acc / Z_H(x), with the Lagrange selectors of
 * vm/src/compiler/recursion/circuit/domain.rs:48-66 (trace domain shift 1).
 * Inputs are the traces' evaluations on the quotient domain
 * GENERATOR * <w_Q>, Q = 2^(log_trace + log_qd), in natural order (Monty
 * form); `prep` or `perm` may be NULL (absent), `perm` rows hold perm_w
 * extension elements (4 words each).  `global` holds the global cumulative
 * sum's 14 coordinates.  out: Q x 4 words (Monty). */
enum {
    ORC_Q_MAIN = 1, ORC_Q_PREP = 2, ORC_Q_PERM = 3, ORC_Q_CONST = 4, ORC_Q_PUBLIC = 5,
    ORC_Q_FIRST = 6, ORC_Q_LAST = 7, ORC_Q_TRANSITION = 8,
    ORC_Q_ADD = 9, ORC_Q_SUB = 10, ORC_Q_MUL = 11,
    ORC_Q_EADD = 12, ORC_Q_ESUB = 13, ORC_Q_EMUL = 14, ORC_Q_EMB = 15, ORC_Q_EMULB = 16,
    ORC_Q_CHALLENGE = 17, ORC_Q_REGIONAL = 18, ORC_Q_GLOBAL = 19,
    ORC_Q_ASSERT = 20, ORC_Q_EASSERT = 21
};
int orc_quotient_values(int field, uint32_t log_trace, uint32_t log_qd, const uint32_t *prep, uint32_t prep_w,
                        const uint32_t *main, uint32_t main_w, const uint32_t *perm, uint32_t perm_w,
                        const uint32_t *ops, uint32_t n_ops, const uint32_t *pub, uint32_t n_pub,
                        const uint32_t *chal, uint32_t n_chal, const uint32_t regional[4],
                        const uint32_t global[14], const uint32_t alpha[4], uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
