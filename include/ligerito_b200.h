/*
 * ligerito_b200.h -- C ABI of liblgpu.so, the B200 (sm_100a) implementation
 * of the Ligerito prover hot path of ashutosh1206/ligerito-rust.
 *
 * Plain C types only: host pointers, device pointers (as plain pointers),
 * sizes.  Every call returns an lg_status and never aborts the process;
 * where the reference panics, the call returns an error status instead.
 * The field is GF(2^32) with x^32 + x^15 + x^9 + x^7 + x^4 + x^3 + 1
 * (src/binary_field.rs:179-181); elements travel as uint32_t.
 *
 * Each declaration names the reference interface it replaces
 * (path:line inside the reference project).
 */
#ifndef LIGERITO_B200_H
#define LIGERITO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LG_ABI_VERSION 1
#define LG_MAX_STEPS 8
#define LG_NUM_QUERIES 148 /* s, src/prover.rs:30 and src/verifier.rs:25 */
#define LG_FS_SEED 1234u   /* src/prover.rs:29 and src/verifier.rs:24 */

typedef enum lg_status {
    LG_OK = 0,
    LG_ERR_INVALID_ARGUMENT = 1, /* null pointer, size out of range */
    LG_ERR_INVALID_CONFIG = 2,   /* config the reference would panic on */
    LG_ERR_OUT_OF_MEMORY = 3,    /* device allocation or HBM budget */
    LG_ERR_CUDA = 4,             /* CUDA runtime error (see lg_ctx_last_error) */
    LG_ERR_VERIFY_PANIC = 5,     /* the reference verifier would have panicked */
    LG_ERR_PROVER_ASSERT = 6,    /* a prover-side assert of the reference failed */
    LG_ERR_NO_DEVICE = 7,        /* no CUDA device / library built without one */
    LG_ERR_MALFORMED_PROOF = 8,  /* proof bytes do not parse */
    LG_ERR_EXCEEDS_STATIC_SCRATCH = 9, /* sizes beyond the fixed scratch of a *_noalloc call */
    LG_ERR_TIMEOUT = 10                /* lg_server_wait: not finished within the timeout */
} lg_status;

/* Mirrors ProverConfig / VerifierConfig (src/data_structures.rs:9-30) without
 * the precomputed Reed-Solomon tables, which the context caches:
 *   initial_dims = (2^initial_log_m, 2^initial_log_n), dims[i] =
 *   (2^log_m[i], 2^log_n[i]), ks[i], initial_k, recursive_steps.
 * The verifier reads initial_dim = initial_log_m and log_dims = log_m. */
typedef struct lg_config {
    uint32_t recursive_steps;
    uint32_t initial_log_m;
    uint32_t initial_log_n;
    uint32_t initial_k;
    uint32_t log_m[LG_MAX_STEPS];
    uint32_t log_n[LG_MAX_STEPS];
    uint32_t ks[LG_MAX_STEPS];
} lg_config;

typedef struct lg_ctx lg_ctx;     /* one device, one stream, caches; one host thread */
typedef struct lg_proof lg_proof; /* FinalizedLigeritoProof<BinaryElem32> */

const char *lg_status_string(lg_status s);
uint32_t lg_abi_version(void);

/* ---------------------------------------------------------------- configs */
/* hardcoded_config_20 / hardcoded_config_20_verifier, src/config.rs:6-67 */
lg_status lg_hardcoded_config_20(lg_config *out);
/* hardcoded_config_24 / hardcoded_config_24_verifier, src/config.rs:69-134 */
lg_status lg_hardcoded_config_24(lg_config *out);
/* Sizes config.rs has no function for (2^16..2^30), by the same pattern:
 * initial (2^(L-6), 2^6) with k = 6, then (2^(d-4), 2^4) steps from
 * d = L-6 while d-4 >= 10; L = 16..19 get one step (2^(L-10), 2^4).
 * Reproduces config 20 and 24 exactly. */
lg_status lg_config_make(uint32_t log_size, lg_config *out);
/* The consistency the reference asserts while proving (src/prover.rs,
 * src/sumcheck_polys.rs:97): LG_OK or LG_ERR_INVALID_CONFIG. */
lg_status lg_config_validate(const lg_config *cfg, uint64_t poly_len);
/* A config as text, in place of the hard-coded ProverConfig values of
 * src/config.rs:6-134: lines "key = values" for recursive_steps,
 * initial_dims (rows columns), initial_k, dims (one "rows columns" pair per
 * step, pairs separated by commas) and ks; '#' starts a comment; every
 * dimension a power of two.  Parse errors are LG_ERR_INVALID_CONFIG; the
 * result still goes through lg_config_validate when proving.  Format writes
 * the same form with its terminating NUL (buf NULL: *len = the size). */
lg_status lg_config_parse(const char *text, lg_config *out);
lg_status lg_config_format(const lg_config *cfg, char *buf, uint64_t *len);

/* ---------------------------------------------------------------- context */
/* hbm_budget_bytes = 0: no budget.  Fails with LG_ERR_NO_DEVICE without a GPU. */
lg_status lg_ctx_create(int device, uint64_t hbm_budget_bytes, lg_ctx **out);
void lg_ctx_destroy(lg_ctx *ctx);
const char *lg_ctx_last_error(const lg_ctx *ctx);
void *lg_ctx_stream(lg_ctx *ctx);        /* the cudaStream_t every call is issued on */
lg_status lg_ctx_synchronize(lg_ctx *ctx);
uint64_t lg_ctx_launch_count(const lg_ctx *ctx); /* kernels this context launched */
/* Autotuning (off by default; LG_AUTOTUNE=1 in the environment turns it on
 * for new contexts): with it on, the first whole FFT of a shape (length,
 * vectors, subtrees) and the first fold of a shape time their candidate
 * stage splits / grids on scratch buffers and keep the fastest for the
 * process, every context of the device.  Every choice gives the same
 * results.  lg_tuned_choices lists the choices made, one per line (buf
 * NULL: *len = the size with its NUL).  No reference counterpart. */
lg_status lg_ctx_set_autotune(lg_ctx *ctx, int enabled);
lg_status lg_tuned_choices(char *buf, uint64_t *len);
/* Per-kernel CUDA-event timing (off by default); stats accumulate until reset. */
lg_status lg_ctx_set_kernel_timing(lg_ctx *ctx, int enabled);
lg_status lg_ctx_kernel_stats(lg_ctx *ctx, uint32_t index, char *name, size_t name_cap,
                              uint64_t *launches, double *total_ms); /* INVALID_ARGUMENT past end */
lg_status lg_ctx_reset_kernel_stats(lg_ctx *ctx);
/* Algorithmic work of the timed launches of entry `index` (the same order as
 * lg_ctx_kernel_stats), summed over its launches: compulsory HBM bytes (every
 * input read once, every output written once), GF(2^32) multiplications and
 * BLAKE3 compressions.  The roofline of each kernel divides these by the
 * device's peak rates.  No reference counterpart (measurement only). */
lg_status lg_ctx_kernel_work(lg_ctx *ctx, uint32_t index, double *hbm_bytes, double *gf_mults,
                             double *blake3_compressions);
uint64_t lg_ctx_device_bytes_in_use(const lg_ctx *ctx);
/* Device bytes a context keeps between calls (its arena, reserved on its
 * first call, and its FFT tables), and the bytes of the code / twiddle
 * tables that all contexts on a device share (ReedSolomonEncoding::new's
 * twiddles and pis per size, src/reed_solomon.rs:49-64), held while a
 * context on that device exists. */
uint64_t lg_ctx_device_bytes_cached(const lg_ctx *ctx);
uint64_t lg_device_table_bytes(int device);

/* Peak rates of the device's integer pipes and shared memory, measured by
 * throughput microkernels on `device`: rates[k] for k < count (k an
 * lg_pipe), in instructions per second over the whole device.  LG_PIPE_LDS
 * counts warp-wide conflict-free shared loads (wavefronts); LG_PIPE_LOP3_IMAD
 * counts both instructions of an interleaved pair, so it shows whether the
 * logic and multiply-add pipes issue together.  These are the denominators of
 * the integer rooflines.  No reference counterpart (measurement only). */
typedef enum lg_pipe {
    LG_PIPE_LOP3 = 0,      /* 3-input logic (XOR) */
    LG_PIPE_IADD = 1,      /* 32-bit add */
    LG_PIPE_PRMT = 2,      /* byte permute */
    LG_PIPE_SHF = 3,       /* funnel shift */
    LG_PIPE_IMAD = 4,      /* 32-bit multiply-add, low half */
    LG_PIPE_IMAD_HI = 5,   /* 32-bit multiply-add, high half */
    LG_PIPE_LOP3_IMAD = 6, /* LOP3 and IMAD interleaved */
    LG_PIPE_LDS = 7,       /* conflict-free 32-bit shared-memory loads */
    LG_PIPE_COUNT = 8
} lg_pipe;
lg_status lg_measure_pipe_peaks(int device, double *rates, uint32_t count);

/* ------------------------------------------------------------ prove/verify */
/* prover::<BinaryElem32>(config, poly), src/prover.rs:15.  `poly` holds
 * `len` coefficients on the host (poly_on_device = 0) or on this context's
 * device (1); the caller keeps ownership.  The Fiat-Shamir seed is 1234 and
 * s = 148 as in the reference.  *out is freed with lg_proof_free. */
lg_status lg_prove(lg_ctx *ctx, const lg_config *cfg, const uint32_t *poly, uint64_t len,
                   int poly_on_device, lg_proof **out);

/* Debug / parity: the same proof as lg_prove, handing each intermediate of
 * src/prover.rs:15-199 to `cb` as soon as the device has produced it (the
 * call synchronises at every one, so it is much slower than lg_prove).
 * `data` is a host copy valid only during the callback.  Names and levels
 * (level = recursion depth of the commitment or opening; round = global
 * sumcheck round; triple = index in the proof's transcript order):
 *   "twiddles" / "pis"      level  ReedSolomonEncoding::new tables, u32
 *                                  (reed_solomon.rs:49-64)
 *   "encoded" / "tree"      level  ligero_commit: column-major encoded
 *                                  matrix (u32) and all Merkle layers,
 *                                  leaves first, 32 B per node (ligero.rs:70-95)
 *   "fold_challenges"       0      the initial_k partial_eval challenges
 *   "folded"                0      partial_eval(poly, challenges) (prover.rs:52-53)
 *   "queries"               level  sorted distinct queries opened on that
 *                                  commitment, u64 (emulated_fs.rs:62-75)
 *   "opened_rows"           level  their rows, row-major u32 (ligero.rs:40-51)
 *   "alpha"                 level  the induce challenge (prover.rs:68,158)
 *   "basis" / "enforced_sum" level induce_sumcheck_poly_parallel's output
 *                                  (sumcheck_polys.rs:83-160)
 *   "triple"                triple (s0, s1, s2) of eval_013 / eval_01x
 *   "round_challenge"       round  the fold challenge of that round
 *   "round_f" / "round_basis" round f and the summed basis after the fold
 *                                  (ligerito.rs:119-127; the reference folds
 *                                  each basis polynomial, whose sum this is)
 *   "beta" / "basis_sum"    level  the glue challenge and the summed basis
 *                                  after glue (ligerito.rs:59-67)
 *   "yr"                    steps  the final folded vector (prover.rs:104-110)
 * *out receives the proof, as lg_prove. */
typedef void (*lg_dump_cb)(void *user, const char *name, uint32_t level, const void *data, uint64_t bytes);
lg_status lg_dump_intermediates(lg_ctx *ctx, const lg_config *cfg, const uint32_t *poly, uint64_t len,
                                int poly_on_device, lg_dump_cb cb, void *user, lg_proof **out);

/* verifier::<BinaryElem32>(config, proof), src/verifier.rs:10.  LG_OK with
 * *accepted = the reference's return value; LG_ERR_VERIFY_PANIC (accepted =
 * 0) where the reference panics (Merkle / Ligero asserts, malformed sizes). */
lg_status lg_verify(lg_ctx *ctx, const lg_config *cfg, const lg_proof *proof, int *accepted);
/* The same from the proof's bytes (lg_proof_serialize's encoding), so a
 * caller holding only bytes needs no parser: LG_ERR_MALFORMED_PROOF when
 * they do not parse, otherwise as lg_verify (verifier.rs:10). */
lg_status lg_verify_bytes(lg_ctx *ctx, const lg_config *cfg, const uint8_t *proof, uint64_t len,
                          int *accepted);

/* Canonical byte encoding in the field order of FinalizedLigeritoProof
 * (src/data_structures.rs:91-103); the reference keeps proofs in memory
 * only.  buf = NULL queries the size into *len. */
lg_status lg_proof_serialize(const lg_proof *proof, uint8_t *buf, uint64_t *len);
lg_status lg_proof_deserialize(const uint8_t *buf, uint64_t len, lg_proof **out);
void lg_proof_free(lg_proof *proof);
/* ProofSize::proof_size, src/data_structures.rs:165-194 */
lg_status lg_proof_size(const lg_proof *proof, uint64_t *bytes);

/* Lockstep batch: `count` polynomials of one config (each `len` words, on
 * the device or all on the host) proved together on one context, up to 64
 * per group, every kernel launch covering the whole group (the proof index
 * is a grid dimension); out[i] is the proof of polys[i], the same bytes
 * lg_prove gives alone.  Device inputs that are already contiguous
 * (polys[i] = polys[0] + i * len) are read in place, others are first
 * copied into one buffer.  A proof whose prover assertion fails gets
 * out[i] = NULL and the call returns LG_ERR_PROVER_ASSERT; other proofs of
 * the call are still returned.  (A loop of src/prover.rs:15 over the
 * polynomials.) */
lg_status lg_prove_lockstep(lg_ctx *ctx, const lg_config *cfg, const uint32_t *const *polys, uint64_t len,
                            uint32_t count, int polys_on_device, lg_proof **out);

/* ------------------------------------------------- batched / served proving
 * Many proofs of uneven sizes on one GPU.  A server runs `workers`
 * threads, each with its own context; requests are admitted FIFO when their
 * device footprint fits hbm_budget_bytes (0 = no budget) next to the ones
 * in flight, and each admitted request is proved by the next free worker,
 * so proofs that arrive while others run start as soon as a worker and
 * memory free up and their GPU work overlaps.  Every proof is the same
 * bytes lg_prove gives alone.  (The reference proves one polynomial per
 * call, src/prover.rs:15; these have no counterpart there.) */
typedef struct lg_server lg_server;
lg_status lg_server_create(int device, uint64_t hbm_budget_bytes, uint32_t workers, lg_server **out);
/* A worker that takes a request also takes up to max_batch - 1 queued
 * requests of the same config and input kind (in queue order, while they
 * fit the budget) and proves them in lockstep (lg_prove_lockstep).
 * 1 (the default) proves one request at a time; at most 64. */
lg_status lg_server_set_max_batch(lg_server *srv, uint32_t max_batch);
/* copy_input = 1 copies a host polynomial so the caller may free it at
 * once; otherwise (and always for device input) it must stay valid until
 * lg_server_wait returns for this ticket. */
lg_status lg_server_submit(lg_server *srv, const lg_config *cfg, const uint32_t *poly, uint64_t len,
                           int poly_on_device, int copy_input, uint64_t *ticket);
/* timeout_ms < 0 waits forever; LG_ERR_TIMEOUT leaves the ticket valid.
 * latency_ms = submit -> done, queue_ms = submit -> start (may be NULL).
 * A ticket's result is handed out once: of several threads waiting on one
 * ticket, the first to wake takes it and the others get
 * LG_ERR_INVALID_ARGUMENT, as does any later wait on it. */
lg_status lg_server_wait(lg_server *srv, uint64_t ticket, int64_t timeout_ms, lg_proof **proof,
                         double *latency_ms, double *queue_ms);
lg_status lg_server_stats(lg_server *srv, uint64_t *completed, uint64_t *queued, uint64_t *in_flight_bytes);
void lg_server_destroy(lg_server *srv); /* finishes queued work first */
/* Proves one polynomial of each of the `count` configs on every worker at
 * once (inputs generated on the device), so that every worker's context has
 * its tables for those sizes and the device memory pool has grown to all
 * workers proving the largest size together: requests that follow pay none
 * of these first-use costs.  Waits for the proofs and discards them. */
lg_status lg_server_warm(lg_server *srv, const lg_config *cfgs, uint32_t count);
/* count proofs on `workers` concurrent contexts, same-config proofs in
 * lockstep groups of up to 8 (lg_server_set_max_batch); out[i] as
 * lg_prove */
lg_status lg_prove_batch(int device, uint32_t workers, const lg_config *cfgs, const uint32_t *const *polys,
                         const uint64_t *lens, int polys_on_device, uint32_t count, lg_proof **out);

/* ----------------------------------------------------- kernel entry points
 * Device pointers belong to the context's device; work is issued on the
 * context stream and these calls return after it completes. */

/* compute_twiddles(log_n, None), src/binary_fft.rs:30-58; host output of
 * 2^log_n - 1 heap-ordered entries (log_n in 1..30). */
lg_status lg_compute_twiddles(uint32_t log_n, uint32_t *out);

/* fft(v, &compute_twiddles(log_n), _), src/binary_fft.rs:4-17, applied in
 * place to `batch` contiguous vectors of 2^log_n elements. */
lg_status lg_fft(lg_ctx *ctx, uint32_t *d_data, uint32_t log_n, uint64_t batch);
/* ifft(v, &compute_twiddles(log_n)), src/binary_fft.rs:19-28, same layout. */
lg_status lg_ifft(lg_ctx *ctx, uint32_t *d_data, uint32_t log_n, uint64_t batch);

/* ReedSolomonEncoding::new(2^log_m, 2^(log_m+2)).encode_non_systematic on
 * every column of poly2flatmat: src/reed_solomon.rs:104-113 with
 * src/ligero.rs:11-38.  d_poly: n columns of 2^log_m (column j at
 * j*2^log_m); d_encoded: n columns of 2^(log_m+2), column-major. */
lg_status lg_rs_encode_cols(lg_ctx *ctx, const uint32_t *d_poly, uint32_t log_m, uint32_t n,
                            uint32_t *d_encoded);

/* ligero_commit, src/ligero.rs:70-95: the encoded matrix (as above) and the
 * BLAKE3 Merkle tree over its rows (src/merkle_tree.rs:22-60, leaves = rows
 * as little-endian bytes, src/ligero.rs:53-68).  d_tree receives all layers
 * leaves first, 32*(2*rows-1) bytes; root (host, 32 bytes) may be NULL. */
lg_status lg_ligero_commit(lg_ctx *ctx, const uint32_t *d_poly, uint32_t log_m, uint32_t n,
                           uint32_t *d_encoded, uint8_t *d_tree, uint8_t *root);

/* MultiLinearPoly::partial_eval(rs), src/multilinear_poly.rs:66-87: folds
 * the top k variables of d_evals (2^log_len) into d_out (2^(log_len-k)). */
lg_status lg_partial_eval(lg_ctx *ctx, const uint32_t *d_evals, uint32_t log_len,
                          const uint32_t *rs, uint32_t k, uint32_t *d_out);

/* eval_013_product(f, g), src/multilinear_poly.rs:90-131 -> out[3] (host). */
lg_status lg_eval_013_product(lg_ctx *ctx, const uint32_t *d_f, const uint32_t *d_g,
                              uint32_t log_len, uint32_t out[3]);

/* induce_sumcheck_poly_parallel, src/sumcheck_polys.rs:74-160: rows are
 * host row-major (nrows x 2^nch), queries sorted; basis into d_basis_out
 * (2^n) and the enforced sum into *enforced_sum. */
lg_status lg_induce_sumcheck_poly(lg_ctx *ctx, uint32_t n, const uint32_t *rows, uint32_t nrows,
                                  const uint32_t *v_challenges, uint32_t nch,
                                  const uint64_t *queries, uint32_t alpha, uint32_t *d_basis_out,
                                  uint32_t *enforced_sum);

/* ------------------------------------------------ host-side protocol parts
 * Fiat-Shamir transcript, FS (src/emulated_fs.rs:6-76): running SHA-256
 * over the seed's LE bytes, absorbed bytes and each squeeze's LE counter. */
typedef struct lg_transcript lg_transcript;
lg_status lg_transcript_new(uint32_t seed, lg_transcript **out);        /* FS::new, :12 */
void lg_transcript_free(lg_transcript *t);
lg_status lg_transcript_absorb(lg_transcript *t, const uint8_t *bytes, uint64_t len); /* :18 */
lg_status lg_transcript_squeeze(lg_transcript *t, uint64_t out[2]);     /* :22, u128 low/high */
lg_status lg_transcript_get_field(lg_transcript *t, uint32_t *out);     /* :34, BinaryElem32 */
lg_status lg_transcript_get_query(lg_transcript *t, uint64_t n, uint64_t *out); /* :56 */
/* :61; LG_ERR_INVALID_ARGUMENT where the reference loops forever (n < s) */
lg_status lg_transcript_get_distinct_queries(lg_transcript *t, uint64_t n, uint64_t s, uint64_t *out);

/* merkle_tree::verify (src/merkle_tree.rs:164-188) with BLAKE3 leaves and
 * nodes: leaf i = leaves[leaf_off[i] .. leaf_off[i+1]], proof = n_sib
 * 32-byte siblings.  LG_OK with *ok = the reference's bool, or
 * LG_ERR_VERIFY_PANIC where it indexes past the proof. */
lg_status lg_merkle_verify(const uint8_t *root, const uint8_t *proof, uint64_t n_sib, uint64_t depth,
                           const uint8_t *leaves, const uint64_t *leaf_off, const uint64_t *queries,
                           uint64_t nq, int *ok);

/* The same result as lg_induce_sumcheck_poly, for callers that cannot
 * allocate device memory: their device memory is owned by another allocator
 * that reserved it up front, or they run on a path that must not call
 * cudaMalloc / cudaFree because those can synchronise the whole device.
 * No counterpart in the reference (it is an allocation-free variant of the
 * call above, not a reference interface).
 *
 * Inputs and outputs are the caller's device buffers: d_rows (nrows x
 * 2^nch words, row-major), d_queries (nrows sorted row indices, each below
 * 2^32: the device reads their low 32 bits, so larger values, which the
 * regular call rejects with LG_ERR_INVALID_ARGUMENT, give undefined
 * results here), d_basis_out (2^n words), d_enforced_sum (1 word);
 * v_challenges stays on the host.  Work is queued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream) behind the work already
 * on it, and the call returns without waiting for it.
 *
 * Scratch comes from one fixed array of LG_NOALLOC_SCRATCH_BYTES in device
 * memory, held by every GPU that has loaded it until the process exits.
 * Limit: nrows <= 256 and n <= 20 (anything larger returns
 * LG_ERR_EXCEEDS_STATIC_SCRATCH and queues no work).  The array lives in
 * its own code module, which the CUDA runtime loads lazily: the first call
 * on each device loads that module and reserves the array there (the
 * driver allocates it, which can synchronise the device) and looks up the
 * array's device address.  Make one warm-up call on each device at
 * start-up, before any stream capture and before latency-critical work;
 * later calls allocate nothing.  All calls share the array: calls whose
 * work overlaps on the GPU race on it, so order them on one stream or wait
 * between them. */
#define LG_NOALLOC_SCRATCH_BYTES (4u << 20)
lg_status lg_induce_sumcheck_poly_noalloc(void *stream, uint32_t n, const uint32_t *d_rows, uint32_t nrows,
                                          const uint32_t *v_challenges, uint32_t nch,
                                          const uint64_t *d_queries, uint32_t alpha, uint32_t *d_basis_out,
                                          uint32_t *d_enforced_sum);

/* BinaryElem128 multiplication (define_galois_field!(BinaryElem128, u128,
 * 0x87, ...), src/binary_field.rs:182-189, with the generic product of
 * :52-105): d_out[i] = d_a[i] * d_b[i] mod x^128 + x^7 + x^2 + x + 1 for n
 * elements, each two little-endian u64 limbs (bits 0-63, then 64-127) in
 * device memory; the arrays must be 16-byte aligned.  The reference prover
 * uses only BinaryElem32; this is the 128-bit field for a 128-bit-challenge
 * variant. */
lg_status lg_gf128_mul(lg_ctx *ctx, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out, uint64_t n);

/* Seeded coefficient generator (SplitMix64; coefficient i = low 32 bits of
 * output i).  The reference draws unseeded rand::random (src/main.rs:25). */
lg_status lg_fill_splitmix(lg_ctx *ctx, uint64_t seed, uint32_t *d_out, uint64_t n);
void lg_fill_splitmix_host(uint64_t seed, uint32_t *out, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif /* LIGERITO_B200_H */
