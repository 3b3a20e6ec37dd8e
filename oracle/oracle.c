/*
 * CPU oracle for the trace-commitment path (test infrastructure only; see
 * oracle.h).  Plain C11 + OpenMP; canonical-form arithmetic with 64-bit `%`.
 *
 * Sources restated (paths relative to the reference repository):
 *   - Poseidon2 constants: vm/src/primitives/mod.rs:37-218 (raw table),
 *     :305-346 (split into external / internal constants), internal diagonal
 *     vm/src/primitives/consts.rs:110-127 (BabyBear), :136-154 (KoalaBear),
 *     round counts and S-box degrees consts.rs:184-203.
 *   - Permutation round structure: gnark/poseidon2/poseidon2_koalabear.go:71-98
 *     (and the BabyBear twin), external layer :126-159, internal layer :162-196.
 *   - Sponge / compression: vm/src/compiler/recursion/circuit/hash.rs:40-52,
 *     :89-94 (TruncatedPermutation fills all 16 lanes with left||right).
 *   - Mixed-height MMCS: vm/src/compiler/recursion/circuit/fri.rs:389-436.
 *   - FRI fold, x coordinates, final polynomial: fri.rs:45-52, :288-387,
 *     :514-521; commit-phase loop of TwoAdicFriPcs::open (prover.rs:589).
 *   - Duplex challenger: vm/src/compiler/recursion/circuit/challenger.rs:89-115,
 *     :202-237.
 *   - Coset generators 3 (KoalaBear) / 31 (BabyBear):
 *     vm/src/compiler/recursion/ir/utils.rs:13-19; LDE shift GENERATOR /
 *     domain.shift and bit-reversed rows: TwoAdicFriPcs::commit as called from
 *     vm/src/machine/prover.rs:102,244,415,540; committed row i <-> x =
 *     g * w_N^rev(i): fri.rs:155-171.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    uint32_t p;
    uint32_t two_adicity;
    uint32_t generator;
    uint32_t w_ext; /* x^4 = W in the degree-4 extension */
    uint32_t sbox_deg;
    uint32_t rounds_p;
    uint32_t diag[16];
    uint32_t rc[30][16]; /* reduced mod p */
} field_t;

static const uint32_t RC_RAW[30][16] = {
#include "../pico_b200/csrc/p2_rc_table.inc"
};

static field_t FIELDS[2];
static int fields_ready = 0;

static void init_fields(void) {
    if (fields_ready) return;
    for (int f = 0; f < 2; f++) {
        field_t *F = &FIELDS[f];
        uint32_t p;
        if (f == ORC_KOALABEAR) {
            p = 0x7f000001u;
            F->two_adicity = 24;
            F->generator = 3;
            F->w_ext = 3;
            F->sbox_deg = 3;
            F->rounds_p = 20;
            uint32_t d[16] = {p - 2, 1, 2, (p + 1) >> 1, 3, 4, (p - 1) >> 1, p - 3, p - 4,
                              p - ((p - 1) >> 8), p - ((p - 1) >> 3), p - 127,
                              (p - 1) >> 8, (p - 1) >> 3, (p - 1) >> 4, 127};
            memcpy(F->diag, d, sizeof d);
        } else {
            p = 0x78000001u;
            F->two_adicity = 27;
            F->generator = 31;
            F->w_ext = 11;
            F->sbox_deg = 7;
            F->rounds_p = 13;
            uint32_t d[16] = {p - 2, 1, 2, (p + 1) >> 1, 3, 4, (p - 1) >> 1, p - 3, p - 4,
                              p - ((p - 1) >> 8), p - ((p - 1) >> 2), p - ((p - 1) >> 3),
                              p - 15, (p - 1) >> 8, (p - 1) >> 4, 15};
            memcpy(F->diag, d, sizeof d);
        }
        F->p = p;
        for (int r = 0; r < 30; r++)
            for (int j = 0; j < 16; j++) F->rc[r][j] = RC_RAW[r][j] % p;
    }
    fields_ready = 1;
}

static const field_t *fld(int field) {
    init_fields();
    return &FIELDS[field == ORC_BABYBEAR ? 1 : 0];
}

/* ---------------- canonical field arithmetic ---------------- */
static inline uint32_t fadd(uint32_t p, uint32_t a, uint32_t b) {
    uint64_t s = (uint64_t)a + b;
    return (uint32_t)(s >= p ? s - p : s);
}
static inline uint32_t fsub(uint32_t p, uint32_t a, uint32_t b) {
    return a >= b ? a - b : a + p - b;
}
static inline uint32_t fmul(uint32_t p, uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * b) % p);
}
static uint32_t fpow(uint32_t p, uint32_t a, uint64_t e) {
    uint32_t r = 1;
    while (e) {
        if (e & 1) r = fmul(p, r, a);
        a = fmul(p, a, a);
        e >>= 1;
    }
    return r;
}
static inline uint32_t finv(uint32_t p, uint32_t a) { return fpow(p, a, p - 2); }

uint32_t orc_prime(int field) { return fld(field)->p; }
uint32_t orc_generator(int field) { return fld(field)->generator; }

uint32_t orc_to_monty(int field, uint32_t x) {
    uint32_t p = fld(field)->p;
    return (uint32_t)((((uint64_t)(x % p)) << 32) % p);
}
uint32_t orc_from_monty(int field, uint32_t x) {
    uint32_t p = fld(field)->p;
    uint32_t rinv = finv(p, (uint32_t)((1ull << 32) % p));
    return fmul(p, x % p, rinv);
}

uint32_t orc_two_adic_generator(int field, uint32_t bits) {
    const field_t *F = fld(field);
    if (bits > F->two_adicity) return 0;
    return fpow(F->p, F->generator, (uint64_t)(F->p - 1) >> bits);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------- Poseidon2-16 (canonical) ---------------- */
/* 4x4 block [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] as the add chain of
 * gnark/poseidon2/poseidon2_koalabear.go:126-136. */
static void m4(uint32_t p, uint32_t *s) {
    uint32_t t01 = fadd(p, s[0], s[1]);
    uint32_t t23 = fadd(p, s[2], s[3]);
    uint32_t t0123 = fadd(p, t01, t23);
    uint32_t t01123 = fadd(p, t0123, s[1]);
    uint32_t t01233 = fadd(p, t0123, s[3]);
    uint32_t n3 = fadd(p, t01233, fadd(p, s[0], s[0]));
    uint32_t n1 = fadd(p, t01123, fadd(p, s[2], s[2]));
    uint32_t n0 = fadd(p, t01123, t01);
    uint32_t n2 = fadd(p, t01233, t23);
    s[0] = n0; s[1] = n1; s[2] = n2; s[3] = n3;
}

static void external_layer(uint32_t p, uint32_t *s) {
    for (int i = 0; i < 16; i += 4) m4(p, s + i);
    uint32_t sums[4];
    for (int k = 0; k < 4; k++) sums[k] = fadd(p, fadd(p, s[k], s[4 + k]), fadd(p, s[8 + k], s[12 + k]));
    for (int i = 0; i < 16; i++) s[i] = fadd(p, s[i], sums[i & 3]);
}

static void internal_layer(const field_t *F, uint32_t *s) {
    uint32_t p = F->p, sum = 0;
    for (int i = 0; i < 16; i++) sum = fadd(p, sum, s[i]);
    for (int i = 0; i < 16; i++) s[i] = fadd(p, fmul(p, s[i], F->diag[i]), sum);
}

static inline uint32_t sbox(const field_t *F, uint32_t x) { return fpow(F->p, x, F->sbox_deg); }

static void permute_canon(const field_t *F, uint32_t *s) {
    uint32_t p = F->p;
    const uint32_t rp = F->rounds_p;
    external_layer(p, s);
    for (uint32_t r = 0; r < 4; r++) {
        for (int j = 0; j < 16; j++) s[j] = sbox(F, fadd(p, s[j], F->rc[r][j]));
        external_layer(p, s);
    }
    for (uint32_t r = 4; r < 4 + rp; r++) {
        s[0] = sbox(F, fadd(p, s[0], F->rc[r][0]));
        internal_layer(F, s);
    }
    for (uint32_t r = 4 + rp; r < 8 + rp; r++) {
        for (int j = 0; j < 16; j++) s[j] = sbox(F, fadd(p, s[j], F->rc[r][j]));
        external_layer(p, s);
    }
}

int orc_permute_canonical(int field, uint32_t state[16]) {
    const field_t *F = fld(field);
    for (int i = 0; i < 16; i++)
        if (state[i] >= F->p) return ORC_EINVAL;
    permute_canon(F, state);
    return ORC_OK;
}

/* Monty <-> canonical helpers with precomputed R^-1 */
typedef struct { uint32_t p, rinv, r; } conv_t;
static conv_t conv(const field_t *F) {
    conv_t c;
    c.p = F->p;
    c.r = (uint32_t)((1ull << 32) % F->p);
    c.rinv = finv(F->p, c.r);
    return c;
}
static inline uint32_t c_from(conv_t c, uint32_t x) { return fmul(c.p, x % c.p, c.rinv); }
static inline uint32_t c_to(conv_t c, uint32_t x) { return fmul(c.p, x, c.r); }

/* Synthetic inputs: SplitMix64 draws >> 33, values >= p skipped (the
 * generator of pico_b200/fields.py uniform()), converted to Monty form. */
void orc_uniform_monty(int field, uint64_t seed, uint64_t n, uint32_t *out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint64_t z0 = seed;
    uint64_t i = 0;
    while (i < n) {
        z0 += 0x9E3779B97F4A7C15ull;
        uint64_t z = z0;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        uint32_t v = (uint32_t)(z >> 33);
        if (v < F->p) out[i++] = c_to(c, v);
    }
}

int orc_permute(int field, uint32_t *states, size_t n) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)n; k++) {
        uint32_t s[16];
        for (int i = 0; i < 16; i++) s[i] = c_from(c, states[16 * k + i]);
        permute_canon(F, s);
        for (int i = 0; i < 16; i++) states[16 * k + i] = c_to(c, s[i]);
    }
    return ORC_OK;
}

/* ---------------- sponge / compression (canonical) ---------------- */
/* PaddingFreeSponge<Perm,16,8,8>: overwrite-mode absorption of 8-element
 * chunks, permute after each chunk (hash.rs:40-52). */
typedef struct {
    uint32_t s[16];
    int pos;
} sponge_t;
static void sponge_init(sponge_t *sp) { memset(sp, 0, sizeof *sp); }
static inline void sponge_absorb(const field_t *F, sponge_t *sp, uint32_t v) {
    sp->s[sp->pos++] = v;
    if (sp->pos == 8) {
        permute_canon(F, sp->s);
        sp->pos = 0;
    }
}
static void sponge_finish(const field_t *F, sponge_t *sp, uint32_t out[8]) {
    if (sp->pos != 0) permute_canon(F, sp->s);
    memcpy(out, sp->s, 8 * sizeof(uint32_t));
}

static void compress_canon(const field_t *F, const uint32_t *l, const uint32_t *r, uint32_t *out) {
    uint32_t s[16];
    memcpy(s, l, 32);
    memcpy(s + 8, r, 32);
    permute_canon(F, s);
    memcpy(out, s, 32);
}

int orc_hash(int field, const uint32_t *in, size_t len, uint32_t out[8]) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    sponge_t sp;
    sponge_init(&sp);
    for (size_t i = 0; i < len; i++) sponge_absorb(F, &sp, c_from(c, in[i]));
    uint32_t d[8];
    sponge_finish(F, &sp, d);
    for (int i = 0; i < 8; i++) out[i] = c_to(c, d[i]);
    return ORC_OK;
}

int orc_compress(int field, const uint32_t left[8], const uint32_t right[8], uint32_t out[8]) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t l[8], r[8], o[8];
    for (int i = 0; i < 8; i++) { l[i] = c_from(c, left[i]); r[i] = c_from(c, right[i]); }
    compress_canon(F, l, r, o);
    for (int i = 0; i < 8; i++) out[i] = c_to(c, o[i]);
    return ORC_OK;
}

/* ---------------- mixed-height MMCS (fri.rs:389-436) ---------------- */
static int is_pow2(uint64_t x) { return x && !(x & (x - 1)); }

/* Hash row `r` of the concatenation of matrices idx[0..k) (canonical digest). */
static void hash_concat_row(const field_t *F, conv_t c, const uint32_t *const *mats,
                            const uint32_t *widths, const uint32_t *idx, uint32_t k,
                            uint64_t r, uint32_t out[8]) {
    sponge_t sp;
    sponge_init(&sp);
    for (uint32_t m = 0; m < k; m++) {
        const uint32_t *row = mats[idx[m]] + r * widths[idx[m]];
        for (uint32_t j = 0; j < widths[idx[m]]; j++) sponge_absorb(F, &sp, c_from(c, row[j]));
    }
    sponge_finish(F, &sp, out);
}

int orc_mmcs_commit(int field, uint32_t n_mats, const uint32_t *const *mats,
                    const uint64_t *heights, const uint32_t *widths,
                    uint32_t root[8], uint32_t *layers) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    if (n_mats == 0) return ORC_EINVAL;
    /* stable sort by height descending (tallest first) */
    uint32_t *order = malloc(n_mats * sizeof(uint32_t));
    if (!order) return ORC_ENOMEM;
    for (uint32_t i = 0; i < n_mats; i++) {
        if (!is_pow2(heights[i])) { free(order); return ORC_EINVAL; }
        order[i] = i;
    }
    for (uint32_t i = 1; i < n_mats; i++) { /* insertion sort: stable */
        uint32_t v = order[i];
        int j = (int)i - 1;
        while (j >= 0 && heights[order[j]] < heights[v]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = v;
    }
    uint64_t hmax = heights[order[0]];
    uint32_t *cur = malloc(hmax * 8 * sizeof(uint32_t));
    uint32_t *nxt = malloc((hmax / 2 + 1) * 8 * sizeof(uint32_t));
    if (!cur || !nxt) { free(order); free(cur); free(nxt); return ORC_ENOMEM; }

    uint32_t gpos = 0, gk = 0;
    while (gpos + gk < n_mats && heights[order[gpos + gk]] == hmax) gk++;
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < (long long)hmax; r++)
        hash_concat_row(F, c, mats, widths, order + gpos, gk, (uint64_t)r, cur + 8 * r);
    gpos += gk;
    size_t loff = 0;
    if (layers) {
        for (uint64_t i = 0; i < hmax * 8; i++) layers[i] = c_to(c, cur[i]);
        loff = hmax * 8;
    }
    uint64_t len = hmax;
    while (len > 1) {
        uint64_t nlen = len / 2;
        gk = 0;
        while (gpos + gk < n_mats && heights[order[gpos + gk]] == nlen) gk++;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)nlen; i++) {
            uint32_t d[8];
            compress_canon(F, cur + 16 * i, cur + 16 * i + 8, d);
            if (gk) {
                uint32_t rd[8];
                hash_concat_row(F, c, mats, widths, order + gpos, gk, (uint64_t)i, rd);
                compress_canon(F, d, rd, d);
            }
            memcpy(nxt + 8 * i, d, 32);
        }
        gpos += gk;
        uint32_t *t = cur; cur = nxt; nxt = t;
        len = nlen;
        if (layers) {
            for (uint64_t i = 0; i < len * 8; i++) layers[loff + i] = c_to(c, cur[i]);
            loff += len * 8;
        }
    }
    for (int i = 0; i < 8; i++) root[i] = c_to(c, cur[i]);
    free(order); free(cur); free(nxt);
    return ORC_OK;
}

/* ---------------- NTT / coset LDE ---------------- */
static inline uint64_t bitrev(uint64_t x, uint32_t bits) {
    uint64_t r = 0;
    for (uint32_t i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* In-place natural-order -> natural-order transform X[k] = sum_j a[j] w^(jk),
 * w a primitive 2^log_n-th root (iterative bit-reversal + Cooley-Tukey). */
static void ntt_inplace(uint32_t p, uint32_t *a, uint32_t log_n, uint32_t w) {
    uint64_t n = 1ull << log_n;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t j = bitrev(i, log_n);
        if (j > i) { uint32_t t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (uint32_t s = 1; s <= log_n; s++) {
        uint64_t m = 1ull << s, h = m >> 1;
        uint32_t wm = fpow(p, w, (1ull << (log_n - s)));
        for (uint64_t k = 0; k < n; k += m) {
            uint32_t t = 1;
            for (uint64_t j = 0; j < h; j++) {
                uint32_t u = a[k + j], v = fmul(p, a[k + j + h], t);
                a[k + j] = fadd(p, u, v);
                a[k + j + h] = fsub(p, u, v);
                t = fmul(p, t, wm);
            }
        }
    }
}

int orc_coset_lde(int field, const uint32_t *in, uint32_t log_n, uint32_t w,
                  uint32_t log_blowup, uint32_t shift_monty, int bitrev_rows,
                  uint32_t *out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t p = F->p;
    uint32_t log_N = log_n + log_blowup;
    if (log_N > F->two_adicity) return ORC_EINVAL;
    uint64_t n = 1ull << log_n, N = 1ull << log_N;
    uint32_t wn = orc_two_adic_generator(field, log_n);
    uint32_t wn_inv = finv(p, wn);
    uint32_t wN = orc_two_adic_generator(field, log_N);
    uint32_t shift = c_from(c, shift_monty);
    uint32_t n_inv = finv(p, (uint32_t)(n % p));
    int err = 0;
#pragma omp parallel
    {
        uint32_t *col = malloc(N * sizeof(uint32_t));
        if (!col) {
#pragma omp atomic write
            err = 1;
        }
#pragma omp for schedule(dynamic)
        for (long long j = 0; j < (long long)w; j++) {
            if (!col) continue;
            for (uint64_t r = 0; r < n; r++) col[r] = c_from(c, in[r * w + j]);
            ntt_inplace(p, col, log_n, wn_inv); /* evaluations -> n * coefficients */
            uint32_t sp = n_inv;
            for (uint64_t r = 0; r < n; r++) { col[r] = fmul(p, col[r], sp); sp = fmul(p, sp, shift); }
            for (uint64_t r = n; r < N; r++) col[r] = 0;
            ntt_inplace(p, col, log_N, wN);
            for (uint64_t r = 0; r < N; r++) {
                uint64_t dst = bitrev_rows ? bitrev(r, log_N) : r;
                out[dst * w + j] = c_to(c, col[r]);
            }
        }
        free(col);
    }
    return err ? ORC_ENOMEM : ORC_OK;
}

int orc_pcs_commit(int field, uint32_t n_mats, const uint32_t *const *mats,
                   const uint32_t *log_heights, const uint32_t *widths,
                   const uint32_t *shifts, uint32_t log_blowup,
                   uint32_t root[8], uint32_t *const *ldes, uint32_t *layers) {
    if (n_mats == 0) return ORC_EINVAL;
    uint32_t **bufs = calloc(n_mats, sizeof(uint32_t *));
    uint64_t *heights = malloc(n_mats * sizeof(uint64_t));
    if (!bufs || !heights) { free(bufs); free(heights); return ORC_ENOMEM; }
    int rc = ORC_OK;
    for (uint32_t m = 0; m < n_mats && rc == ORC_OK; m++) {
        uint64_t N = 1ull << (log_heights[m] + log_blowup);
        heights[m] = N;
        bufs[m] = (ldes && ldes[m]) ? ldes[m] : malloc(N * (uint64_t)widths[m] * sizeof(uint32_t) + 4);
        if (!bufs[m]) { rc = ORC_ENOMEM; break; }
        rc = orc_coset_lde(field, mats[m], log_heights[m], widths[m], log_blowup, shifts[m], 1, bufs[m]);
    }
    if (rc == ORC_OK)
        rc = orc_mmcs_commit(field, n_mats, (const uint32_t *const *)bufs, heights, widths, root, layers);
    for (uint32_t m = 0; m < n_mats; m++)
        if (!(ldes && ldes[m])) free(bufs[m]);
    free(bufs);
    free(heights);
    return rc;
}

/* ---------------- challenger (challenger.rs:89-115, 202-237) ---------------- */
void orc_challenger_init(orc_challenger *ch) { memset(ch, 0, sizeof *ch); }

static void duplexing(const field_t *F, conv_t c, orc_challenger *ch) {
    uint32_t s[16];
    for (uint32_t i = 0; i < ch->in_len; i++) ch->sponge[i] = ch->in_buf[i];
    ch->in_len = 0;
    for (int i = 0; i < 16; i++) s[i] = c_from(c, ch->sponge[i]);
    permute_canon(F, s);
    for (int i = 0; i < 16; i++) ch->sponge[i] = c_to(c, s[i]);
    for (int i = 0; i < 8; i++) ch->out_buf[i] = ch->sponge[i];
    ch->out_len = 8;
}

void orc_challenger_observe(int field, orc_challenger *ch, uint32_t v) {
    const field_t *F = fld(field);
    ch->out_len = 0;
    ch->in_buf[ch->in_len++] = v;
    if (ch->in_len == 8) duplexing(F, conv(F), ch);
}

uint32_t orc_challenger_sample(int field, orc_challenger *ch) {
    const field_t *F = fld(field);
    if (ch->in_len != 0 || ch->out_len == 0) duplexing(F, conv(F), ch);
    return ch->out_buf[--ch->out_len];
}

/* ---------------- extension field (x^4 = W) ---------------- */
static void ext_mul_c(uint32_t p, uint32_t W, const uint32_t *a, const uint32_t *b, uint32_t *o) {
    uint64_t acc[7] = {0};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) acc[i + j] = (acc[i + j] + (uint64_t)a[i] * b[j]) % p;
    for (int k = 0; k < 4; k++) {
        uint64_t v = acc[k];
        if (k + 4 < 7) v = (v + (acc[k + 4] % p) * W) % p;
        o[k] = (uint32_t)v;
    }
}

void orc_ext_mul(int field, const uint32_t a[4], const uint32_t b[4], uint32_t out[4]) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t x[4], y[4], z[4];
    for (int i = 0; i < 4; i++) { x[i] = c_from(c, a[i]); y[i] = c_from(c, b[i]); }
    ext_mul_c(F->p, F->w_ext, x, y, z);
    for (int i = 0; i < 4; i++) out[i] = c_to(c, z[i]);
}

/* ---------------- FRI commit phase ---------------- */
/*
 * One fold (TwoAdicFriGenericConfig::fold_matrix as mirrored by the verifier,
 * fri.rs:345-377): rows r of the (len/2) x 2 matrix (lo, hi) fold to
 *   (1/2 + beta/2 * g_inv^rev(r)) * lo + (1/2 - beta/2 * g_inv^rev(r)) * hi,
 * g = two_adic_generator(log len), rev over log(len/2) bits.  This equals the
 * verifier's e0 + (beta - x0)(e1 - e0)/(x1 - x0) with x1 = -x0.
 */
static void fri_fold(const field_t *F, const uint32_t *cw, uint64_t len, const uint32_t *beta,
                     uint32_t *out) {
    uint32_t p = F->p;
    uint32_t log_len = 0;
    while ((1ull << log_len) < len) log_len++;
    uint64_t h = len / 2;
    uint32_t g_inv = finv(p, fpow(p, F->generator, (uint64_t)(p - 1) >> log_len));
    uint32_t half = finv(p, 2);
    uint32_t hb[4];
    for (int i = 0; i < 4; i++) hb[i] = fmul(p, beta[i], half);
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < (long long)h; r++) {
        uint32_t gp = fpow(p, g_inv, bitrev((uint64_t)r, log_len - 1));
        uint32_t pw[4], a[4], b[4];
        for (int i = 0; i < 4; i++) pw[i] = fmul(p, hb[i], gp);
        for (int i = 0; i < 4; i++) {
            a[i] = pw[i];
            b[i] = fsub(p, 0, pw[i]);
        }
        a[0] = fadd(p, a[0], half);
        b[0] = fadd(p, b[0], half);
        uint32_t t1[4], t2[4];
        ext_mul_c(p, F->w_ext, a, cw + 8 * r, t1);
        ext_mul_c(p, F->w_ext, b, cw + 8 * r + 4, t2);
        for (int i = 0; i < 4; i++) out[4 * r + i] = fadd(p, t1[i], t2[i]);
    }
}

int orc_fri_commit_phase(int field, const uint32_t *codeword, uint32_t log_n,
                         uint32_t log_blowup, uint32_t log_final_len,
                         const uint32_t *betas_in, orc_challenger *ch,
                         uint32_t *roots, uint32_t *betas, uint32_t *final_out,
                         uint32_t *rounds_out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t p = F->p;
    uint32_t log_stop = log_blowup + log_final_len;
    if (log_n < log_stop || log_n > F->two_adicity) return ORC_EINVAL;
    uint64_t len = 1ull << log_n;
    uint32_t *cur = malloc(len * 4 * sizeof(uint32_t));
    uint32_t *nxt = malloc((len / 2 + 1) * 4 * sizeof(uint32_t));
    if (!cur || !nxt) { free(cur); free(nxt); return ORC_ENOMEM; }
    for (uint64_t i = 0; i < len * 4; i++) cur[i] = c_from(c, codeword[i]);
    uint32_t round = 0;
    while (len > (1ull << log_stop)) {
        /* commit the (len/2) x 2 extension matrix, flattened to 8 base columns */
        uint64_t h = len / 2;
        uint32_t *mono = malloc(len * 4 * sizeof(uint32_t));
        if (!mono) { free(cur); free(nxt); return ORC_ENOMEM; }
        for (uint64_t i = 0; i < len * 4; i++) mono[i] = c_to(c, cur[i]);
        const uint32_t *mats[1] = {mono};
        uint64_t hh[1] = {h};
        uint32_t ww[1] = {8};
        uint32_t root[8];
        int rc = orc_mmcs_commit(field, 1, mats, hh, ww, root, NULL);
        free(mono);
        if (rc) { free(cur); free(nxt); return rc; }
        if (roots) memcpy(roots + 8 * round, root, 32);
        uint32_t beta[4];
        if (betas_in) {
            for (int i = 0; i < 4; i++) beta[i] = betas_in[4 * round + i];
        } else {
            for (int i = 0; i < 8; i++) orc_challenger_observe(field, ch, root[i]);
            for (int i = 0; i < 4; i++) beta[i] = orc_challenger_sample(field, ch);
        }
        if (betas) memcpy(betas + 4 * round, beta, 16);
        uint32_t bc[4];
        for (int i = 0; i < 4; i++) bc[i] = c_from(c, beta[i]);
        fri_fold(F, cur, len, bc, nxt);
        uint32_t *t = cur; cur = nxt; nxt = t;
        len = h;
        round++;
    }
    if (log_final_len == 0) {
        /* Plonky3 final_poly: the remaining 2^b evaluations are all equal */
        for (uint64_t i = 1; i < len; i++)
            for (int k = 0; k < 4; k++)
                if (cur[4 * i + k] != cur[k]) { free(cur); free(nxt); return ORC_EINVAL; }
        if (final_out)
            for (int k = 0; k < 4; k++) final_out[k] = c_to(c, cur[k]);
        if (!betas_in)
            for (int k = 0; k < 4; k++) orc_challenger_observe(field, ch, c_to(c, cur[k]));
    } else {
        /* Coefficients of the final polynomial: the remaining codeword holds
         * evaluations on the subgroup H_len in bit-reversed order (the fold
         * ignores the coset shift); un-permute, inverse transform, keep the
         * first 2^log_final_len coefficients. */
        uint32_t log_len = log_stop;
        uint32_t *nat = malloc(len * 4 * sizeof(uint32_t));
        uint32_t *colv = malloc(len * sizeof(uint32_t));
        if (!nat || !colv) { free(nat); free(colv); free(cur); free(nxt); return ORC_ENOMEM; }
        for (uint64_t i = 0; i < len; i++)
            for (int k = 0; k < 4; k++) nat[4 * bitrev(i, log_len) + k] = cur[4 * i + k];
        uint32_t winv = finv(p, orc_two_adic_generator(field, log_len));
        uint32_t linv = finv(p, (uint32_t)(len % p));
        uint64_t keep = 1ull << log_final_len;
        for (int k = 0; k < 4; k++) {
            for (uint64_t i = 0; i < len; i++) colv[i] = nat[4 * i + k];
            ntt_inplace(p, colv, log_len, winv);
            for (uint64_t i = 0; i < len; i++) {
                uint32_t v = fmul(p, colv[i], linv);
                if (i < keep) {
                    if (final_out) final_out[4 * i + k] = c_to(c, v);
                } else if (v != 0) {
                    free(nat); free(colv); free(cur); free(nxt);
                    return ORC_EINVAL;
                }
            }
        }
        free(nat);
        free(colv);
        if (!betas_in)
            for (uint64_t i = 0; i < keep; i++)
                for (int k = 0; k < 4; k++) orc_challenger_observe(field, ch, final_out ? final_out[4 * i + k] : 0);
    }
    if (rounds_out) *rounds_out = round;
    free(cur);
    free(nxt);
    return ORC_OK;
}

/* ===================== PCS opening (TwoAdicFriPcs::open) =====================
 * The prover side of the opening, restated from what the Pico verifier checks
 * (every step below is fixed by vm/src/compiler/recursion/circuit/fri.rs):
 *   - every opened value is observed (its 4 base coefficients, in batch /
 *     matrix / point / column order) before alpha is sampled: fri.rs:85-99;
 *   - reduced openings per LDE height, with the powers of alpha counted per
 *     height in that same order and x = g * w_h^rev(index): fri.rs:113-238;
 *   - the FRI commit phase folds the tallest reduced opening and adds each
 *     shorter one once the folded length reaches its height: fri.rs:300-318;
 *   - the final polynomial is observed, the proof-of-work witness checked and
 *     the query indices sampled: fri.rs:54-70 (check_witness / sample_bits:
 *     challenger.rs:109-115, 210-221);
 *   - query openings: an MMCS batch opening of every input batch
 *     (fri.rs:389-436) and the commit-phase sibling values and paths
 *     (fri.rs:320-343).
 * Opened values follow Plonky3's interpolate_coset: barycentric evaluation
 * over the low coset g * H_n held in the first n rows of each committed LDE.
 */

static void ext_add_c(uint32_t p, const uint32_t *a, const uint32_t *b, uint32_t *o) {
    for (int i = 0; i < 4; i++) o[i] = fadd(p, a[i], b[i]);
}
static void ext_sub_c(uint32_t p, const uint32_t *a, const uint32_t *b, uint32_t *o) {
    for (int i = 0; i < 4; i++) o[i] = fsub(p, a[i], b[i]);
}
static void ext_scale_c(uint32_t p, const uint32_t *a, uint32_t s, uint32_t *o) {
    for (int i = 0; i < 4; i++) o[i] = fmul(p, a[i], s);
}
static void ext_pow_c(const field_t *F, const uint32_t *a, uint64_t e, uint32_t *o) {
    uint32_t r[4] = {1, 0, 0, 0}, b[4];
    memcpy(b, a, 16);
    while (e) {
        if (e & 1) ext_mul_c(F->p, F->w_ext, r, b, r);
        ext_mul_c(F->p, F->w_ext, b, b, b);
        e >>= 1;
    }
    memcpy(o, r, 16);
}
/* Inverse through the norm to F_p: a^-1 = a^p a^(p^2) a^(p^3) / N(a).  With
 * X^4 = W the Frobenius maps X to gamma X, gamma = W^((p-1)/4), so the k-th
 * conjugate multiplies coefficient i by gamma^(k i). */
static void ext_inv_c(const field_t *F, const uint32_t *a, uint32_t *o) {
    uint32_t p = F->p;
    uint32_t gamma = fpow(p, F->w_ext, (p - 1) / 4);
    uint32_t c1[4], c2[4], c3[4], t[4], n[4];
    for (int i = 0; i < 4; i++) {
        c1[i] = fmul(p, a[i], fpow(p, gamma, (uint64_t)i));
        c2[i] = fmul(p, a[i], fpow(p, gamma, 2ull * i));
        c3[i] = fmul(p, a[i], fpow(p, gamma, 3ull * i));
    }
    ext_mul_c(p, F->w_ext, c1, c2, t);
    ext_mul_c(p, F->w_ext, t, c3, t);
    ext_mul_c(p, F->w_ext, a, t, n); /* n[1..3] == 0 */
    ext_scale_c(p, t, finv(p, n[0]), o);
}

void orc_ext_inv(int field, const uint32_t a[4], uint32_t out[4]) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t x[4], y[4];
    for (int i = 0; i < 4; i++) x[i] = c_from(c, a[i]);
    ext_inv_c(F, x, y);
    for (int i = 0; i < 4; i++) out[i] = c_to(c, y[i]);
}

/* g * w_h^rev_h(i), canonical. */
static uint32_t lde_point(const field_t *F, uint32_t wh, uint32_t log_h, uint64_t i) {
    return fmul(F->p, F->generator, fpow(F->p, wh, bitrev(i, log_h)));
}

/* p(z) for every column of one matrix (interpolate_coset); z and out canonical. */
static int open_one(const field_t *F, conv_t c, int field, const uint32_t *lde, uint32_t log_N, uint32_t w,
                    uint32_t log_b, const uint32_t *z, uint32_t *out) {
    uint32_t p = F->p;
    uint32_t log_n = log_N - log_b;
    uint64_t n = 1ull << log_n;
    uint32_t *coef = malloc(n * 16);
    if (!coef) return ORC_ENOMEM;
    uint32_t wn = orc_two_adic_generator(field, log_n);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)n; k++) {
        uint32_t wk = fpow(p, wn, (uint64_t)k);
        uint32_t d[4];
        memcpy(d, z, 16);
        d[0] = fsub(p, d[0], fmul(p, F->generator, wk));
        uint32_t di[4];
        ext_inv_c(F, d, di);
        ext_scale_c(p, di, wk, coef + 4 * k);
    }
    /* (z^n - g^n) / (n g^(n-1)) */
    uint32_t zn[4], s[4];
    ext_pow_c(F, z, n, zn);
    zn[0] = fsub(p, zn[0], fpow(p, F->generator, n));
    uint32_t den = fmul(p, (uint32_t)(n % p), fpow(p, F->generator, n - 1));
    ext_scale_c(p, zn, finv(p, den), s);
#pragma omp parallel for schedule(static)
    for (long long j = 0; j < (long long)w; j++) {
        uint32_t acc[4] = {0, 0, 0, 0}, t[4];
        for (uint64_t k = 0; k < n; k++) {
            /* natural index k sits at bit-reversed position rev(k) of the prefix */
            uint32_t y = c_from(c, lde[bitrev(k, log_n) * w + (uint64_t)j]);
            ext_scale_c(p, coef + 4 * k, y, t);
            ext_add_c(p, acc, t, acc);
        }
        ext_mul_c(p, F->w_ext, acc, s, out + 4 * j);
    }
    free(coef);
    return ORC_OK;
}

static uint64_t batch_value_words(const orc_open_batch *b) {
    uint64_t v = 0;
    for (uint32_t m = 0; m < b->n_mats; m++) v += 4ull * b->n_points[m] * b->widths[m];
    return v;
}

int orc_open_values(int field, const orc_open_batch *b, uint32_t log_blowup, uint32_t *values) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    const uint32_t *pt = b->points;
    uint32_t *out = values;
    for (uint32_t m = 0; m < b->n_mats; m++) {
        if (b->log_heights[m] < log_blowup) return ORC_EINVAL;
        for (uint32_t k = 0; k < b->n_points[m]; k++, pt += 4) {
            uint32_t z[4];
            for (int i = 0; i < 4; i++) z[i] = c_from(c, pt[i]);
            uint32_t *o = malloc((uint64_t)b->widths[m] * 16 + 16);
            if (!o) return ORC_ENOMEM;
            int rc = open_one(F, c, field, b->ldes[m], b->log_heights[m], b->widths[m], log_blowup, z, o);
            if (rc) { free(o); return rc; }
            for (uint64_t i = 0; i < 4ull * b->widths[m]; i++) out[i] = c_to(c, o[i]);
            out += 4ull * b->widths[m];
            free(o);
        }
    }
    return ORC_OK;
}

/* Reduced openings: ro[h] (2^h x 4, canonical) for every LDE height h of a
 * matrix, zero where no point is opened; alpha canonical, values Monty. */
static int reduce_openings(const field_t *F, conv_t c, int field, const orc_open_batch *batches,
                           uint32_t n_batches, const uint32_t *values, const uint32_t *alpha, uint32_t **ro) {
    uint32_t p = F->p;
    uint64_t num_reduced[32] = {0};
    /* distinct points and the tallest height each is opened at */
    uint32_t n_pts = 0, cap = 16;
    uint32_t (*pts)[4] = malloc(cap * 16);
    uint32_t *pt_log = malloc(cap * 4);
    uint32_t **dinv = NULL;
    int rc = ORC_OK;
    if (!pts || !pt_log) { rc = ORC_ENOMEM; goto out; }
    for (uint32_t b = 0; b < n_batches; b++) {
        const uint32_t *pt = batches[b].points;
        for (uint32_t m = 0; m < batches[b].n_mats; m++)
            for (uint32_t k = 0; k < batches[b].n_points[m]; k++, pt += 4) {
                uint32_t z[4];
                for (int i = 0; i < 4; i++) z[i] = c_from(c, pt[i]);
                uint32_t q = 0;
                while (q < n_pts && memcmp(pts[q], z, 16) != 0) q++;
                if (q == n_pts) {
                    if (n_pts == cap) {
                        cap *= 2;
                        void *a = realloc(pts, cap * 16), *l = realloc(pt_log, cap * 4);
                        if (a) pts = a;
                        if (l) pt_log = l;
                        if (!a || !l) { rc = ORC_ENOMEM; goto out; }
                    }
                    memcpy(pts[q], z, 16);
                    pt_log[q] = 0;
                    n_pts++;
                }
                if (batches[b].log_heights[m] > pt_log[q]) pt_log[q] = batches[b].log_heights[m];
            }
    }
    /* 1 / (z - x_i) over the tallest height of each point; shorter heights use
     * a prefix (bit-reversed order nests the subgroups). */
    dinv = calloc(n_pts ? n_pts : 1, sizeof(uint32_t *));
    if (!dinv) { rc = ORC_ENOMEM; goto out; }
    for (uint32_t q = 0; q < n_pts; q++) {
        uint64_t N = 1ull << pt_log[q];
        dinv[q] = malloc(N * 16);
        if (!dinv[q]) { rc = ORC_ENOMEM; goto out; }
        uint32_t wh = orc_two_adic_generator(field, pt_log[q]);
        const uint32_t *z = pts[q];
        uint32_t *dq = dinv[q];
        uint32_t lq = pt_log[q];
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; i++) {
            uint32_t d[4];
            memcpy(d, z, 16);
            d[0] = fsub(p, d[0], lde_point(F, wh, lq, (uint64_t)i));
            ext_inv_c(F, d, dq + 4 * i);
        }
    }
    const uint32_t *val = values;
    for (uint32_t b = 0; b < n_batches; b++) {
        const orc_open_batch *B = &batches[b];
        const uint32_t *pt = B->points;
        for (uint32_t m = 0; m < B->n_mats; m++) {
            uint32_t h = B->log_heights[m], w = B->widths[m];
            uint64_t N = 1ull << h;
            if (!ro[h]) {
                ro[h] = calloc(N * 4, sizeof(uint32_t));
                if (!ro[h]) { rc = ORC_ENOMEM; goto out; }
            }
            if (B->n_points[m] == 0) continue;
            /* alpha^j for the row reduction */
            uint32_t *apow = malloc(((uint64_t)w + 1) * 16);
            uint32_t *rr = malloc(N * 16);
            if (!apow || !rr) { free(apow); free(rr); rc = ORC_ENOMEM; goto out; }
            apow[0] = 1; apow[1] = apow[2] = apow[3] = 0;
            for (uint32_t j = 1; j <= w; j++) ext_mul_c(p, F->w_ext, apow + 4 * (j - 1), alpha, apow + 4 * j);
            const uint32_t *M = B->ldes[m];
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)N; i++) {
                uint32_t acc[4] = {0, 0, 0, 0}, t[4];
                for (uint32_t j = 0; j < w; j++) {
                    ext_scale_c(p, apow + 4 * j, c_from(c, M[(uint64_t)i * w + j]), t);
                    ext_add_c(p, acc, t, acc);
                }
                memcpy(rr + 4 * i, acc, 16);
            }
            for (uint32_t k = 0; k < B->n_points[m]; k++, pt += 4) {
                uint32_t z[4], rys[4] = {0, 0, 0, 0}, aoff[4], t[4];
                for (int i = 0; i < 4; i++) z[i] = c_from(c, pt[i]);
                uint32_t q = 0;
                while (memcmp(pts[q], z, 16) != 0) q++;
                for (uint32_t j = 0; j < w; j++) {
                    uint32_t y[4];
                    for (int i = 0; i < 4; i++) y[i] = c_from(c, val[4 * j + i]);
                    ext_mul_c(p, F->w_ext, apow + 4 * j, y, t);
                    ext_add_c(p, rys, t, rys);
                }
                ext_pow_c(F, alpha, num_reduced[h], aoff);
                const uint32_t *dq = dinv[q];
                uint32_t *roh = ro[h];
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)N; i++) {
                    uint32_t u[4];
                    ext_sub_c(p, rys, rr + 4 * i, u);
                    ext_mul_c(p, F->w_ext, u, aoff, u);
                    ext_mul_c(p, F->w_ext, u, dq + 4 * i, u);
                    ext_add_c(p, roh + 4 * i, u, roh + 4 * i);
                }
                num_reduced[h] += w;
                val += 4ull * w;
            }
            free(apow);
            free(rr);
        }
    }
out:
    if (dinv)
        for (uint32_t q = 0; q < n_pts; q++) free(dinv[q]);
    free(dinv);
    free(pts);
    free(pt_log);
    return rc;
}

int orc_reduce_openings(int field, const orc_open_batch *batches, uint32_t n_batches, const uint32_t *values,
                        const uint32_t alpha[4], uint32_t log_height, uint32_t *ro_out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t *ro[32] = {0}, a[4];
    for (int i = 0; i < 4; i++) a[i] = c_from(c, alpha[i]);
    int rc = reduce_openings(F, c, field, batches, n_batches, values, a, ro);
    if (rc == ORC_OK) {
        if (log_height >= 32 || !ro[log_height]) rc = ORC_EINVAL;
        else
            for (uint64_t i = 0; i < (4ull << log_height); i++) ro_out[i] = c_to(c, ro[log_height][i]);
    }
    for (int h = 0; h < 32; h++) free(ro[h]);
    return rc;
}

static uint32_t batch_log_max(const orc_open_batch *b) {
    uint32_t l = 0;
    for (uint32_t m = 0; m < b->n_mats; m++) if (b->log_heights[m] > l) l = b->log_heights[m];
    return l;
}

uint64_t orc_open_query_words(const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup) {
    uint32_t log_max = 0;
    uint64_t q = 0;
    for (uint32_t b = 0; b < n_batches; b++) {
        uint32_t lb = batch_log_max(&batches[b]);
        if (lb > log_max) log_max = lb;
        for (uint32_t m = 0; m < batches[b].n_mats; m++) q += batches[b].widths[m];
        q += 8ull * lb;
    }
    for (uint32_t L = log_max; L > log_blowup; L--) q += 4 + 8ull * (L - 1);
    return q;
}

/* First witness w (ascending) with sample_bits(bits) == 0 after observing it. */
static uint32_t grind(int field, const orc_challenger *ch, uint32_t bits) {
    const field_t *F = fld(field);
    const uint32_t mask = (bits >= 32) ? 0xffffffffu : ((1u << bits) - 1u);
    const uint32_t chunk = 1u << 14;
    uint8_t *ok = malloc(chunk);
    if (!ok) return 0xffffffffu;
    for (uint64_t base = 0; base < F->p; base += chunk) {
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < (long long)chunk; k++) {
            uint64_t w = base + (uint64_t)k;
            ok[k] = 0;
            if (w >= F->p) continue;
            orc_challenger t = *ch;
            orc_challenger_observe(field, &t, orc_to_monty(field, (uint32_t)w));
            uint32_t v = orc_from_monty(field, orc_challenger_sample(field, &t));
            ok[k] = (v & mask) == 0;
        }
        for (uint32_t k = 0; k < chunk; k++)
            if (ok[k]) { free(ok); return (uint32_t)(base + k); }
    }
    free(ok);
    return 0xffffffffu;
}

static void observe_ext_monty(int field, orc_challenger *ch, const uint32_t *v) {
    for (int i = 0; i < 4; i++) orc_challenger_observe(field, ch, v[i]);
}
static void sample_ext_monty(int field, orc_challenger *ch, uint32_t *v) {
    for (int i = 0; i < 4; i++) v[i] = orc_challenger_sample(field, ch);
}

int orc_pcs_open(int field, const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup,
                 uint32_t num_queries, uint32_t pow_bits, orc_challenger *ch, uint32_t *values,
                 uint32_t *roots, uint32_t *betas, uint32_t final_poly[4], uint32_t *pow_witness,
                 uint32_t *indices, uint32_t *queries, uint32_t *rounds_out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t p = F->p;
    if (n_batches == 0) return ORC_EINVAL;
    uint32_t log_max = 0;
    for (uint32_t b = 0; b < n_batches; b++) {
        if (batches[b].n_mats == 0) return ORC_EINVAL;
        uint32_t lb = batch_log_max(&batches[b]);
        if (lb > log_max) log_max = lb;
    }
    if (log_max <= log_blowup || log_max > F->two_adicity) return ORC_EINVAL;
    /* 1. opened values, observed in order; alpha */
    uint64_t voff = 0;
    for (uint32_t b = 0; b < n_batches; b++) {
        int rc = orc_open_values(field, &batches[b], log_blowup, values + voff);
        if (rc) return rc;
        voff += batch_value_words(&batches[b]);
    }
    for (uint64_t i = 0; i < voff; i++) orc_challenger_observe(field, ch, values[i]);
    uint32_t alpha[4], ac[4];
    sample_ext_monty(field, ch, alpha);
    for (int i = 0; i < 4; i++) ac[i] = c_from(c, alpha[i]);
    /* 2. reduced openings */
    uint32_t *ro[32] = {0};
    int rc = reduce_openings(F, c, field, batches, n_batches, values, ac, ro);
    uint32_t R = log_max - log_blowup;
    uint32_t **cws = calloc(R + 1, sizeof(uint32_t *)), **lay = calloc(R + 1, sizeof(uint32_t *));
    if (!rc && (!cws || !lay)) rc = ORC_ENOMEM;
    /* 3. commit phase */
    uint32_t *cur = NULL;
    if (!rc) {
        uint64_t len = 1ull << log_max;
        cur = malloc(len * 16);
        if (!cur) rc = ORC_ENOMEM;
        else memcpy(cur, ro[log_max], len * 16);
        for (uint32_t r = 0; !rc && r < R; r++) {
            uint64_t h = len / 2;
            cws[r] = malloc(len * 16);
            lay[r] = malloc((2 * h - 1) * 32);
            uint32_t *nxt = malloc(h * 16);
            if (!cws[r] || !lay[r] || !nxt) { free(nxt); rc = ORC_ENOMEM; break; }
            for (uint64_t i = 0; i < len * 4; i++) cws[r][i] = c_to(c, cur[i]);
            const uint32_t *mats[1] = {cws[r]};
            uint64_t hh[1] = {h};
            uint32_t ww[1] = {8};
            uint32_t root[8], beta[4], bc[4];
            rc = orc_mmcs_commit(field, 1, mats, hh, ww, root, lay[r]);
            if (rc) { free(nxt); break; }
            if (roots) memcpy(roots + 8 * r, root, 32);
            for (int i = 0; i < 8; i++) orc_challenger_observe(field, ch, root[i]);
            sample_ext_monty(field, ch, beta);
            if (betas) memcpy(betas + 4 * r, beta, 16);
            for (int i = 0; i < 4; i++) bc[i] = c_from(c, beta[i]);
            fri_fold(F, cur, len, bc, nxt);
            free(cur);
            cur = nxt;
            len = h;
            uint32_t lh = log_max - r - 1;
            if (ro[lh])
                for (uint64_t i = 0; i < len * 4; i++) cur[i] = fadd(p, cur[i], ro[lh][i]);
        }
        if (!rc) {
            for (uint64_t i = 1; i < len && !rc; i++)
                if (memcmp(cur + 4 * i, cur, 16) != 0) rc = ORC_EINVAL; /* not of low degree */
        }
        if (!rc) {
            uint32_t fm[4];
            for (int i = 0; i < 4; i++) fm[i] = c_to(c, cur[i]);
            if (final_poly) memcpy(final_poly, fm, 16);
            observe_ext_monty(field, ch, fm);
        }
    }
    /* 4. proof of work, query indices */
    if (!rc) {
        uint32_t w = grind(field, ch, pow_bits);
        if (w == 0xffffffffu) rc = ORC_EINVAL;
        else {
            if (pow_witness) *pow_witness = orc_to_monty(field, w);
            orc_challenger_observe(field, ch, orc_to_monty(field, w));
            (void)orc_challenger_sample(field, ch);
        }
    }
    uint64_t qw = orc_open_query_words(batches, n_batches, log_blowup);
    for (uint32_t q = 0; !rc && q < num_queries; q++) {
        uint32_t v = orc_from_monty(field, orc_challenger_sample(field, ch));
        uint64_t idx = v & (uint32_t)((1ull << log_max) - 1);
        if (indices) indices[q] = (uint32_t)idx;
        if (!queries) continue;
        uint32_t *rec = queries + q * qw;
        for (uint32_t b = 0; b < n_batches; b++) {
            const orc_open_batch *B = &batches[b];
            uint32_t lb = batch_log_max(B);
            uint64_t ib = idx >> (log_max - lb);
            for (uint32_t m = 0; m < B->n_mats; m++) {
                uint64_t row = ib >> (lb - B->log_heights[m]);
                memcpy(rec, B->ldes[m] + row * B->widths[m], 4ull * B->widths[m]);
                rec += B->widths[m];
            }
            uint64_t loff = 0;
            for (uint32_t l = 0; l < lb; l++) {
                uint64_t sib = (ib >> l) ^ 1;
                memcpy(rec, B->layers + (loff + sib) * 8, 32);
                rec += 8;
                loff += 1ull << (lb - l);
            }
        }
        for (uint32_t r = 0; r < R; r++) {
            uint32_t L = log_max - r;
            uint64_t ir = idx >> r;
            memcpy(rec, cws[r] + (ir ^ 1) * 4, 16);
            rec += 4;
            uint64_t pair = ir >> 1, loff = 0;
            for (uint32_t l = 0; l + 1 < L; l++) {
                uint64_t sib = (pair >> l) ^ 1;
                memcpy(rec, lay[r] + (loff + sib) * 8, 32);
                rec += 8;
                loff += 1ull << (L - 1 - l);
            }
        }
    }
    if (rounds_out) *rounds_out = R;
    free(cur);
    if (cws) for (uint32_t r = 0; r <= R; r++) free(cws[r]);
    if (lay) for (uint32_t r = 0; r <= R; r++) free(lay[r]);
    free(cws);
    free(lay);
    for (int h = 0; h < 32; h++) free(ro[h]);
    return rc;
}

/* ---------------- verifier (fri.rs:77-436), for tests ---------------- */
/* verify_batch (fri.rs:389-436): rows in input order, canonical digests. */
static int verify_batch_c(const field_t *F, conv_t c, const uint32_t *root_monty, uint32_t n,
                          const uint32_t *log_heights, const uint32_t *widths, const uint32_t *const *rows,
                          uint64_t index, const uint32_t *path, uint32_t path_len) {
    uint32_t order[64];
    if (n == 0 || n > 64) return 0;
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    for (uint32_t i = 1; i < n; i++) {
        uint32_t v = order[i];
        int j = (int)i - 1;
        while (j >= 0 && log_heights[order[j]] < log_heights[v]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = v;
    }
    uint32_t pos = 0, cur_h = log_heights[order[0]];
    sponge_t sp;
    sponge_init(&sp);
    while (pos < n && log_heights[order[pos]] == cur_h) {
        for (uint32_t j = 0; j < widths[order[pos]]; j++) sponge_absorb(F, &sp, c_from(c, rows[order[pos]][j]));
        pos++;
    }
    uint32_t d[8];
    sponge_finish(F, &sp, d);
    for (uint32_t l = 0; l < path_len; l++) {
        uint32_t sib[8];
        for (int i = 0; i < 8; i++) sib[i] = c_from(c, path[8 * l + i]);
        if ((index >> l) & 1) compress_canon(F, sib, d, d);
        else compress_canon(F, d, sib, d);
        cur_h--;
        if (pos < n && log_heights[order[pos]] == cur_h) {
            sponge_init(&sp);
            while (pos < n && log_heights[order[pos]] == cur_h) {
                for (uint32_t j = 0; j < widths[order[pos]]; j++)
                    sponge_absorb(F, &sp, c_from(c, rows[order[pos]][j]));
                pos++;
            }
            uint32_t rd[8];
            sponge_finish(F, &sp, rd);
            compress_canon(F, d, rd, d);
        }
    }
    for (int i = 0; i < 8; i++)
        if (c_to(c, d[i]) != root_monty[i]) return 0;
    return 1;
}

int orc_verify_open(int field, const orc_open_batch *batches, uint32_t n_batches, uint32_t log_blowup,
                    uint32_t num_queries, uint32_t pow_bits, orc_challenger *ch, const uint32_t *values,
                    const uint32_t *roots, uint32_t n_rounds, const uint32_t final_poly[4], uint32_t pow_witness,
                    const uint32_t *queries, uint32_t *indices_out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    uint32_t p = F->p;
    uint64_t nv = 0;
    for (uint32_t b = 0; b < n_batches; b++) nv += batch_value_words(&batches[b]);
    for (uint64_t i = 0; i < nv; i++) orc_challenger_observe(field, ch, values[i]);
    uint32_t alpha[4], beta[64][4];
    sample_ext_monty(field, ch, alpha);
    if (n_rounds > 64) return ORC_EINVAL;
    for (uint32_t r = 0; r < n_rounds; r++) {
        for (int i = 0; i < 8; i++) orc_challenger_observe(field, ch, roots[8 * r + i]);
        sample_ext_monty(field, ch, beta[r]);
    }
    observe_ext_monty(field, ch, final_poly);
    orc_challenger_observe(field, ch, pow_witness);
    uint32_t pw = orc_from_monty(field, orc_challenger_sample(field, ch));
    if (pow_bits && (pw & ((1u << pow_bits) - 1u))) return 10; /* proof of work */
    uint32_t log_max = n_rounds + log_blowup;
    uint32_t ac[4], fc[4];
    for (int i = 0; i < 4; i++) { ac[i] = c_from(c, alpha[i]); fc[i] = c_from(c, final_poly[i]); }
    uint64_t qw = orc_open_query_words(batches, n_batches, log_blowup);
    for (uint32_t q = 0; q < num_queries; q++) {
        uint64_t idx = orc_from_monty(field, orc_challenger_sample(field, ch)) & (uint32_t)((1ull << log_max) - 1);
        if (indices_out) indices_out[q] = (uint32_t)idx;
        const uint32_t *rec = queries + q * qw;
        uint32_t ro[32][4];
        memset(ro, 0, sizeof ro);
        uint32_t pow_h[32] = {0};
        const uint32_t *val = values;
        for (uint32_t b = 0; b < n_batches; b++) {
            const orc_open_batch *B = &batches[b];
            uint32_t lb = batch_log_max(B);
            if (B->n_mats > 64) return ORC_EINVAL;
            const uint32_t *rows[64];
            for (uint32_t m = 0; m < B->n_mats; m++) { rows[m] = rec; rec += B->widths[m]; }
            uint64_t ib = idx >> (log_max - lb);
            if (!verify_batch_c(F, c, B->root, B->n_mats, B->log_heights, B->widths, rows, ib, rec, lb))
                return 11; /* input batch opening */
            rec += 8ull * lb;
            const uint32_t *pt = B->points;
            for (uint32_t m = 0; m < B->n_mats; m++) {
                uint32_t h = B->log_heights[m];
                uint64_t ih = idx >> (log_max - h);
                uint32_t x = lde_point(F, orc_two_adic_generator(field, h), h, ih);
                for (uint32_t k = 0; k < B->n_points[m]; k++, pt += 4) {
                    uint32_t acc[4] = {0, 0, 0, 0}, z[4], t[4], ap[4];
                    for (uint32_t j = 0; j < B->widths[m]; j++) {
                        for (int i = 0; i < 4; i++) t[i] = c_from(c, val[4 * j + i]);
                        t[0] = fsub(p, t[0], c_from(c, rows[m][j]));
                        ext_pow_c(F, ac, pow_h[h]++, ap);
                        ext_mul_c(p, F->w_ext, t, ap, t);
                        ext_add_c(p, acc, t, acc);
                    }
                    val += 4ull * B->widths[m];
                    for (int i = 0; i < 4; i++) z[i] = c_from(c, pt[i]);
                    z[0] = fsub(p, z[0], x);
                    ext_inv_c(F, z, z);
                    ext_mul_c(p, F->w_ext, acc, z, t);
                    ext_add_c(p, ro[h], t, ro[h]);
                }
            }
        }
        if (ro[log_blowup][0] | ro[log_blowup][1] | ro[log_blowup][2] | ro[log_blowup][3]) return 12;
        /* verify_query (fri.rs:288-387) */
        uint32_t folded[4] = {0, 0, 0, 0};
        uint32_t x = fpow(p, orc_two_adic_generator(field, log_max), bitrev(idx, log_max));
        for (uint32_t r = 0; r < n_rounds; r++) {
            uint32_t lf = log_max - 1 - r;
            ext_add_c(p, folded, ro[lf + 1], folded);
            uint32_t bit = (uint32_t)((idx >> r) & 1);
            uint32_t sib[4], e0[4], e1[4];
            for (int i = 0; i < 4; i++) sib[i] = c_from(c, rec[i]);
            rec += 4;
            if (bit) { memcpy(e0, sib, 16); memcpy(e1, folded, 16); }
            else { memcpy(e0, folded, 16); memcpy(e1, sib, 16); }
            uint32_t row[8], lh[1] = {lf}, wd[1] = {8};
            for (int i = 0; i < 4; i++) { row[i] = c_to(c, e0[i]); row[4 + i] = c_to(c, e1[i]); }
            const uint32_t *rp[1] = {row};
            if (!verify_batch_c(F, c, roots + 8 * r, 1, lh, wd, rp, idx >> (r + 1), rec, lf)) return 13;
            rec += 8ull * lf;
            uint32_t x0 = bit ? fsub(p, 0, x) : x, x1 = bit ? x : fsub(p, 0, x);
            uint32_t d[4], bm[4];
            ext_sub_c(p, e1, e0, d);
            ext_scale_c(p, d, finv(p, fsub(p, x1, x0)), d);
            for (int i = 0; i < 4; i++) bm[i] = c_from(c, beta[r][i]);
            bm[0] = fsub(p, bm[0], x0);
            ext_mul_c(p, F->w_ext, bm, d, d);
            ext_add_c(p, e0, d, folded);
            x = fmul(p, x, x);
        }
        if (memcmp(folded, fc, 16) != 0) return 14;
    }
    return ORC_OK;
}

/* ---------------- compute_quotient_values ---------------- */
/* The prover's quotient computation (vm/src/machine/utils.rs:201-350): per
 * point x = GENERATOR * w_Q^i of the quotient domain, the chip's constraints
 * are folded into acc (acc = acc * alpha + c for every assertion, in program
 * order: ProverConstraintFolder::assert_zero / assert_zero_ext,
 * vm/src/machine/folder.rs:223-227,321-327) over the local row i and the next
 * row i + 2^log_qd (cyclically), and the quotient is acc * inv_zerofier.
 * Selectors for the trace domain H = <w_n> (shift 1), from the verifier's
 * restatement vm/src/compiler/recursion/circuit/domain.rs:48-66:
 *   Z_H(x) = x^n - 1, is_first_row = Z_H(x) / (x - 1),
 *   is_last_row = Z_H(x) / (x - w_n^-1), is_transition = x - w_n^-1,
 *   inv_zerofier = 1 / Z_H(x).
 * Canonical arithmetic with Fermat inverses: no batching tricks. */
#define ORC_QB 64
#define ORC_QE 16
int orc_quotient_values(int field, uint32_t log_trace, uint32_t log_qd, const uint32_t *prep, uint32_t prep_w,
                        const uint32_t *main, uint32_t main_w, const uint32_t *perm, uint32_t perm_w,
                        const uint32_t *ops, uint32_t n_ops, const uint32_t *pub, uint32_t n_pub,
                        const uint32_t *chal, uint32_t n_chal, const uint32_t regional[4],
                        const uint32_t global[14], const uint32_t alpha[4], uint32_t *out) {
    const field_t *F = fld(field);
    conv_t c = conv(F);
    const uint32_t p = F->p, W = F->w_ext;
    const uint32_t log_q = log_trace + log_qd;
    if (log_q > F->two_adicity || !main || !ops || !alpha || !out) return ORC_EINVAL;
    const uint64_t Q = 1ull << log_q, n = 1ull << log_trace;
    /* validate the program once */
    for (uint32_t k = 0; k < n_ops; k++) {
        const uint32_t *o = ops + 4 * k;
        const uint32_t op = o[0], d = o[1], a = o[2], b = o[3];
        int ok = 1;
        switch (op) {
        case ORC_Q_MAIN: ok = d < ORC_QB && a < main_w && b <= 1; break;
        case ORC_Q_PREP: ok = d < ORC_QB && prep && a < prep_w && b <= 1; break;
        case ORC_Q_PERM: ok = d < ORC_QE && perm && a < perm_w && b <= 1; break;
        case ORC_Q_CONST: ok = d < ORC_QB; break;
        case ORC_Q_PUBLIC: ok = d < ORC_QB && a < n_pub; break;
        case ORC_Q_FIRST: case ORC_Q_LAST: case ORC_Q_TRANSITION: ok = d < ORC_QB; break;
        case ORC_Q_ADD: case ORC_Q_SUB: case ORC_Q_MUL: ok = d < ORC_QB && a < ORC_QB && b < ORC_QB; break;
        case ORC_Q_EADD: case ORC_Q_ESUB: case ORC_Q_EMUL: ok = d < ORC_QE && a < ORC_QE && b < ORC_QE; break;
        case ORC_Q_EMB: ok = d < ORC_QE && a < ORC_QB; break;
        case ORC_Q_EMULB: ok = d < ORC_QE && a < ORC_QE && b < ORC_QB; break;
        case ORC_Q_CHALLENGE: ok = d < ORC_QE && a < n_chal; break;
        case ORC_Q_REGIONAL: ok = d < ORC_QE && regional; break;
        case ORC_Q_GLOBAL: ok = d < ORC_QB && a < 14 && global; break;
        case ORC_Q_ASSERT: ok = a < ORC_QB; break;
        case ORC_Q_EASSERT: ok = a < ORC_QE; break;
        default: ok = 0;
        }
        if (!ok) return ORC_EINVAL;
    }
    const uint32_t wq = orc_two_adic_generator(field, log_q);
    const uint32_t wn_inv = finv(p, orc_two_adic_generator(field, log_trace));
    const uint32_t g = F->generator;
    uint32_t al[4];
    for (int i = 0; i < 4; i++) al[i] = c_from(c, alpha[i]);
    int err = 0;
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < (long long)Q; ii++) {
        const uint64_t i = (uint64_t)ii, inext = (i + (1ull << log_qd)) & (Q - 1);
        const uint32_t x = fmul(p, g, fpow(p, wq, i));
        const uint32_t zh = fsub(p, fpow(p, x, n), 1);
        const uint32_t sel_first = fmul(p, zh, finv(p, fsub(p, x, 1)));
        const uint32_t sel_last = fmul(p, zh, finv(p, fsub(p, x, wn_inv)));
        const uint32_t sel_trans = fsub(p, x, wn_inv);
        const uint32_t inv_zh = finv(p, zh);
        uint32_t rb[ORC_QB] = {0}, re[ORC_QE][4] = {{0}}, acc[4] = {0, 0, 0, 0};
        for (uint32_t k = 0; k < n_ops; k++) {
            const uint32_t *o = ops + 4 * k;
            const uint32_t op = o[0], d = o[1], a = o[2], b = o[3];
            const uint64_t row = b ? inext : i;
            uint32_t t[4];
            switch (op) {
            case ORC_Q_MAIN: rb[d] = c_from(c, main[row * main_w + a]); break;
            case ORC_Q_PREP: rb[d] = c_from(c, prep[row * prep_w + a]); break;
            case ORC_Q_PERM:
                for (int j = 0; j < 4; j++) re[d][j] = c_from(c, perm[row * 4 * perm_w + 4 * a + j]);
                break;
            case ORC_Q_CONST: rb[d] = c_from(c, a); break;
            case ORC_Q_PUBLIC: rb[d] = c_from(c, pub[a]); break;
            case ORC_Q_FIRST: rb[d] = sel_first; break;
            case ORC_Q_LAST: rb[d] = sel_last; break;
            case ORC_Q_TRANSITION: rb[d] = sel_trans; break;
            case ORC_Q_ADD: rb[d] = fadd(p, rb[a], rb[b]); break;
            case ORC_Q_SUB: rb[d] = fsub(p, rb[a], rb[b]); break;
            case ORC_Q_MUL: rb[d] = fmul(p, rb[a], rb[b]); break;
            case ORC_Q_EADD: for (int j = 0; j < 4; j++) t[j] = fadd(p, re[a][j], re[b][j]); memcpy(re[d], t, 16); break;
            case ORC_Q_ESUB: for (int j = 0; j < 4; j++) t[j] = fsub(p, re[a][j], re[b][j]); memcpy(re[d], t, 16); break;
            case ORC_Q_EMUL: ext_mul_c(p, W, re[a], re[b], t); memcpy(re[d], t, 16); break;
            case ORC_Q_EMB: re[d][0] = rb[a]; re[d][1] = re[d][2] = re[d][3] = 0; break;
            case ORC_Q_EMULB: for (int j = 0; j < 4; j++) t[j] = fmul(p, re[a][j], rb[b]); memcpy(re[d], t, 16); break;
            case ORC_Q_CHALLENGE: for (int j = 0; j < 4; j++) re[d][j] = c_from(c, chal[4 * a + j]); break;
            case ORC_Q_REGIONAL: for (int j = 0; j < 4; j++) re[d][j] = c_from(c, regional[j]); break;
            case ORC_Q_GLOBAL: rb[d] = c_from(c, global[a]); break;
            case ORC_Q_ASSERT:
                ext_mul_c(p, W, acc, al, t);
                t[0] = fadd(p, t[0], rb[a]);
                memcpy(acc, t, 16);
                break;
            case ORC_Q_EASSERT:
                ext_mul_c(p, W, acc, al, t);
                for (int j = 0; j < 4; j++) acc[j] = fadd(p, t[j], re[a][j]);
                break;
            default:
#pragma omp atomic write
                err = 1;
            }
        }
        for (int j = 0; j < 4; j++) out[4 * i + j] = c_to(c, fmul(p, acc[j], inv_zh));
    }
    return err ? ORC_EINVAL : ORC_OK;
}
