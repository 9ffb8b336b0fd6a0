// Host-side pieces of liblgpu: GF(2^32) scalar arithmetic, the SHA-256
// Fiat-Shamir transcript, BLAKE3, configs, proof encoding, Merkle index
// logic and the per-code setup tables.  Everything here is small, serial
// work the protocol keeps on the host; the bulk work is in lg_kernels.cu.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ligerito_b200.h"

namespace lg {

// ---------------------------------------------------------------- GF(2^32)
// x^32 = x^15 + x^9 + x^7 + x^4 + x^3 + 1 (src/binary_field.rs:179-181).
constexpr uint32_t kPolyTail = 0x8299u;

uint32_t gf_mul(uint32_t a, uint32_t b);
uint32_t gf_pow(uint32_t a, uint64_t e);
uint32_t gf_inv(uint32_t a);  // a != 0
inline uint32_t gf_mulx(uint32_t a) { return (a << 1) ^ ((a >> 31) ? kPolyTail : 0u); }

// ------------------------------------------------------------------ SHA-256
struct Sha256 {
    uint32_t h[8];
    uint8_t buf[64];
    uint64_t total = 0;
    size_t n = 0;
    Sha256();
    void update(const uint8_t *p, size_t len);
    void finish(uint8_t out[32]) const;  // digest of a copy; state unchanged
};

// Fiat-Shamir transcript of src/emulated_fs.rs:6-76.
struct Transcript {
    Sha256 h;
    uint32_t counter = 0;
    explicit Transcript(uint32_t seed);
    void absorb(const void *p, size_t len);
    void absorb_u32s(const uint32_t *v, size_t n);  // to_bytes of each, LE
    std::array<uint64_t, 2> squeeze();               // low, high 64 bits of the u128
    uint32_t get_field() { return (uint32_t)squeeze()[0]; }
    uint64_t get_query(uint64_t n) { return squeeze_lo() % n; }
    uint64_t squeeze_lo();  // squeeze()[0] without the high half or the byte round trip
    // rejection of repeats, then sorted; false where the reference loops forever
    bool get_distinct_queries(uint64_t n, size_t s, std::vector<uint64_t> &out);
};

// ------------------------------------------------------------------- BLAKE3
void blake3_hash(const uint8_t *msg, size_t len, uint8_t out[32]);

// ------------------------------------------------------------------ configs
lg_status config_check(const lg_config &c, uint64_t poly_len);

// -------------------------------------------------------------------- proof
// A list of byte strings (a Vec<Vec<u8>>) in one buffer: entry i is
// data[off[i], off[i+1]).  Proofs hold thousands of 32-byte Merkle nodes;
// one allocation for all of them instead of one each.
struct ByteList {
    std::vector<uint8_t> data;
    std::vector<uint64_t> off = {0};
    size_t size() const { return off.size() - 1; }
    const uint8_t *ptr(size_t i) const { return data.data() + off[i]; }
    size_t len(size_t i) const { return off[i + 1] - off[i]; }
    void clear() { data.clear(); off.assign(1, 0); }
    void push(const uint8_t *p, size_t n) {
        data.insert(data.end(), p, p + n);
        off.push_back(data.size());
    }
    // count entries of `each` bytes, back to back at p
    void assign_fixed(const uint8_t *p, size_t count, size_t each) {
        data.assign(p, p + count * each);
        off.resize(count + 1);
        for (size_t i = 0; i <= count; ++i) off[i] = i * each;
    }
};
// The same for a list of u32 rows (a Vec<Vec<u32>>): row i is
// data[off[i], off[i+1]).
struct WordList {
    std::vector<uint32_t> data;
    std::vector<uint64_t> off = {0};
    size_t size() const { return off.size() - 1; }
    const uint32_t *ptr(size_t i) const { return data.data() + off[i]; }
    size_t len(size_t i) const { return off[i + 1] - off[i]; }
    void clear() { data.clear(); off.assign(1, 0); }
    void push(const uint32_t *p, size_t n) {
        data.insert(data.end(), p, p + n);
        off.push_back(data.size());
    }
    // count rows of `each` words, back to back at p
    void assign_fixed(const uint32_t *p, size_t count, size_t each) {
        data.assign(p, p + count * each);
        off.resize(count + 1);
        for (size_t i = 0; i <= count; ++i) off[i] = i * each;
    }
};
struct Opening {
    WordList rows;    // opened_rows
    ByteList merkle;  // merkle_proof
};
struct Proof {  // FinalizedLigeritoProof, src/data_structures.rs:91-103
    std::vector<uint8_t> initial_root;
    std::vector<std::vector<uint8_t>> recursive_roots;
    Opening initial;
    std::vector<Opening> recursive;
    std::vector<uint32_t> yr;
    Opening final_;
    std::vector<std::array<uint32_t, 3>> transcript;
};
std::vector<uint8_t> serialize(const Proof &p);
size_t serialized_size(const Proof &p);
bool deserialize(const uint8_t *buf, size_t len, Proof &p);
uint64_t proof_size(const Proof &p);  // ProofSize, src/data_structures.rs:105-194

// ----------------------------------------------------------- Merkle indices
// Node (layer, index) of every sibling merkle_tree::prove pushes, in order
// (src/merkle_tree.rs:62-111).  queries sorted and distinct.
struct NodeRef { uint32_t layer; uint64_t index; };
void merkle_proof_nodes(const std::vector<uint64_t> &queries, uint64_t num_leaves,
                        std::vector<NodeRef> &out);
// merkle_tree::verify over precomputed leaf hashes (src/merkle_tree.rs:120-188).
// Returns false where the reference would panic (proof index out of range);
// *ok receives the reference's bool otherwise.
bool merkle_verify(const uint8_t *root, size_t root_len,
                   const ByteList &proof, size_t depth,
                   std::vector<std::array<uint8_t, 32>> layer, std::vector<uint64_t> queries,
                   bool *ok);

// ------------------------------------------------------------- setup tables
// compute_twiddles(log_n, None) (src/binary_fft.rs:30-58).  Every layer the
// reference builds is GF(2)-linear in its index (leaf layer 2u, next_s is
// s^2 + c*s, then a scalar), so each layer is filled from its basis by XOR.
void compute_twiddles(uint32_t log_n, uint32_t *out);
// eval_sk_at_vks (src/binary_fft.rs:217-246): log2(n)+1 values
std::vector<uint32_t> eval_sk_at_vks(uint64_t n);
// compute_pis (src/binary_fft.rs:303-322)
void compute_pis(uint64_t m, const std::vector<uint32_t> &sks, uint32_t *out);
// evaluate_lagrange_basis (src/utils.rs:4-27): rs[0] is the index MSB
std::vector<uint32_t> lagrange_basis(const uint32_t *rs, size_t k);
// next_s (src/binary_fft.rs:100-107)
inline uint32_t next_s(uint32_t s, uint32_t c) { return gf_mul(s, s) ^ gf_mul(c, s); }

void splitmix_fill(uint64_t seed, uint32_t *out, uint64_t n, uint64_t first_index = 0);

}  // namespace lg
