/*
 * lgref -- CPU restatement of the Ligerito prover/verifier of
 * ashutosh1206/ligerito-rust (crate `cryptoutils`), used ONLY as test
 * infrastructure: the parity oracle for the CUDA path and the timed CPU
 * baseline.  Nothing in the shipped library links or calls it.
 *
 * Every function cites the reference file:line it restates.  Field
 * arithmetic keeps the reference's bit-serial multiply
 * (src/binary_field.rs:52-105) so the timed baseline has the reference's
 * cost profile; parallel loops sit where the reference uses rayon.
 *
 * Third-party algorithms the reference calls but does not vendor are
 * restated from their public specifications:
 *   - blake3 1.8.2 (Cargo.lock) -> BLAKE3 spec (hash mode, 7 rounds)
 *   - sha2 0.10.9               -> FIPS 180-4 SHA-256
 * Parity pins: the GF(2^16) twiddle KAT (src/binary_fft.rs:330-349), the
 * Merkle root and multi-proof KATs (src/merkle_tree.rs:195-255, which are
 * SHA-256 values: replayed with the hash set to SHA-256), plus Python
 * hashlib / blake3 cross-checks of both hashes in tests/.
 */
#ifndef LGREF_H
#define LGREF_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (panic = the reference would have panicked) ---- */
enum { LGREF_OK = 0, LGREF_PANIC = 1, LGREF_BAD_ARG = 2, LGREF_OOM = 3 };

/* ---- fields: src/binary_field.rs:176-189 ---- */
uint32_t lgref_gf_mul(int bits, uint32_t a, uint32_t b);     /* bits = 16 or 32 */
uint32_t lgref_gf_pow(int bits, uint32_t a, uint64_t e);
int lgref_gf_inv(int bits, uint32_t a, uint32_t *out);       /* PANIC on zero */
void lgref_gf128_mul(const uint64_t a[2], const uint64_t b[2], uint64_t out[2]);
int lgref_gf128_inv(const uint64_t a[2], uint64_t out[2]);

/* ---- additive FFT: src/binary_fft.rs ---- */
void lgref_compute_twiddles(int bits, int log_n, uint32_t *out /* 2^log_n - 1 */);
void lgref_fft(int bits, uint32_t *v, size_t n, const uint32_t *tw, int nthreads);
void lgref_ifft(int bits, uint32_t *v, size_t n, const uint32_t *tw);
void lgref_eval_sk_at_vks(int bits, size_t n, uint32_t *out /* log2(n)+1 */);
void lgref_evaluate_basis(int bits, size_t basis_len, const uint32_t *sks_vks,
                          uint32_t x, uint32_t *out);
void lgref_compute_pis(int bits, size_t pis_len, const uint32_t *sks_vks, uint32_t *out);

/* ---- Reed-Solomon: src/reed_solomon.rs ---- */
void lgref_short_from_long_tw(const uint32_t *l_tw, int n, int k, uint32_t *s_tw);
int lgref_rs_encode(int bits, const uint32_t *msg, size_t msg_len, size_t block_len,
                    uint32_t *out /* block_len */);
int lgref_rs_encode_non_systematic(int bits, uint32_t *v, size_t msg_len, size_t block_len,
                                   int nthreads);

/* ---- hashes (public specifications) ---- */
void lgref_sha256(const uint8_t *msg, size_t len, uint8_t out[32]);
void lgref_blake3(const uint8_t *msg, size_t len, uint8_t out[32]);

/* ---- Merkle tree: src/merkle_tree.rs ---- */
/* Hash used for leaves and nodes: the reference code uses BLAKE3; its own
   Merkle KATs are SHA-256 values (see lgref.c), so both are selectable. */
enum { LGREF_HASH_BLAKE3 = 0, LGREF_HASH_SHA256 = 1 };
/* Leaves given as one buffer plus offsets (leaf i = buf[off[i] .. off[i+1])).
   tree_out holds all layers, leaves first: 32*(2*num_leaves-1) bytes. */
int lgref_merkle_build(int hash_kind, const uint8_t *buf, const size_t *off, size_t num_leaves,
                       uint8_t *tree_out);
/* Multi-proof; *n_sib receives the sibling count, sib_out needs 32*cap bytes. */
int lgref_merkle_prove(const uint8_t *tree, size_t num_leaves, const size_t *queries,
                       size_t nq, uint8_t *sib_out, size_t cap, size_t *n_sib);
int lgref_merkle_verify(int hash_kind, const uint8_t root[32], const uint8_t *sibs,
                        size_t n_sib, size_t depth, const uint8_t *buf, const size_t *off,
                        const size_t *queries, size_t nq, int *ok);

/* ---- Ligero: src/ligero.rs ---- */
/* Encoded matrix column-major (column j = out[j*4m .. (j+1)*4m]) and tree. */
int lgref_ligero_commit(const uint32_t *poly, size_t m, size_t n, uint32_t *flat_out,
                        uint8_t *tree_out, int nthreads);
int lgref_ligero_verify(const size_t *queries, const uint32_t *rows, size_t nrows,
                        size_t row_len, const uint32_t *yr, size_t yr_len,
                        const uint32_t *challenges, size_t nch);

/* ---- multilinear / sumcheck helpers ---- */
void lgref_lagrange_basis(const uint32_t *rs, size_t k, uint32_t *out /* 2^k */);
int lgref_partial_eval(const uint32_t *evals, size_t len, const uint32_t *rs, size_t k,
                       uint32_t *out /* len >> k */, int nthreads);
void lgref_eval_013_product(const uint32_t *f, const uint32_t *g, size_t len, uint32_t out[3]);
int lgref_induce_sumcheck_poly(size_t n, const uint32_t *sks_vks, const uint32_t *rows,
                               size_t nrows, size_t row_len, const uint32_t *v_ch, size_t nch,
                               const size_t *queries, uint32_t alpha, uint32_t *basis_out,
                               uint32_t *enforced_sum, int nthreads);
void lgref_quadratic_from_evals(uint32_t at0, uint32_t at1, uint32_t atx, uint32_t abc[3]);

/* ---- Fiat-Shamir: src/emulated_fs.rs ---- */
typedef struct lgref_fs lgref_fs;
lgref_fs *lgref_fs_new(uint32_t seed);
void lgref_fs_free(lgref_fs *fs);
void lgref_fs_absorb(lgref_fs *fs, const uint8_t *b, size_t len);
void lgref_fs_squeeze(lgref_fs *fs, uint64_t out_le[2]);
uint32_t lgref_fs_get_field32(lgref_fs *fs);
uint64_t lgref_fs_get_query(lgref_fs *fs, uint64_t n);
int lgref_fs_get_distinct_queries(lgref_fs *fs, uint64_t n, size_t s, size_t *out);

/* ---- configs: src/config.rs (20/24) + the size generator for others ---- */
#define LGREF_MAX_STEPS 8
typedef struct {
    uint32_t recursive_steps;
    uint32_t initial_log_m;     /* initial_dims.0 = 2^initial_log_m */
    uint32_t initial_log_n;     /* initial_dims.1 = 2^initial_log_n */
    uint32_t initial_k;
    uint32_t log_m[LGREF_MAX_STEPS];
    uint32_t log_n[LGREF_MAX_STEPS];
    uint32_t ks[LGREF_MAX_STEPS];
} lgref_config;
int lgref_config_make(uint32_t log_size, lgref_config *cfg);

/* ---- prover / verifier: src/prover.rs, src/verifier.rs ---- */
/* The proof travels as its canonical byte encoding (see lgref.c). */
int lgref_prove(const lgref_config *cfg, const uint32_t *poly, size_t len, int nthreads,
                uint8_t **proof_out, size_t *proof_len);
void lgref_free(void *p);
/* *accepted = the reference's bool; returns PANIC where the reference panics */
int lgref_verify(const lgref_config *cfg, const uint8_t *proof, size_t len, int nthreads,
                 int *accepted);

/* Optional trace of the last lgref_prove on this thread (debug/parity). */
typedef struct {
    uint8_t roots[LGREF_MAX_STEPS + 1][32];
    uint32_t n_roots;
    uint32_t challenges[256];
    uint32_t n_challenges;
    uint32_t enforced_sums[LGREF_MAX_STEPS + 1];
    uint32_t n_sums;
} lgref_trace;
void lgref_last_trace(lgref_trace *out);
/* Test hook (negative tests only): bit 0 = flip s2 of the final sumcheck
   round; applies to later lgref_prove calls on this thread. */
void lgref_set_tamper(int flags);

/* ---- seeded input generator (ours; the reference draws unseeded) ---- */
void lgref_splitmix_coeffs(uint64_t seed, uint32_t *out, size_t n);

#ifdef __cplusplus
}
#endif
#endif
