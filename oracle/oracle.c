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
