// oracle/blake3_spec.h -- TEST INFRASTRUCTURE (the oracle). BLAKE3 (unkeyed hash, 32-byte
// output) written from the published BLAKE3 specification (O'Connor, Aumasson, Neves,
// Wilcox-O'Hearn, 2020): the compression function (7 rounds of the ChaCha-derived G over a
// 16-word state), 1024-byte chunks of 64-byte blocks with CHUNK_START / CHUNK_END flags, and a
// binary tree of PARENT nodes whose left subtrees hold the largest power of two of chunks.
// The reference hashes each tick's state with the `blake3` crate 1.8.2 (Cargo.lock:267-269,
// riftphys-core/src/hash.rs:1-21); that crate is not vendored, so this restatement is pinned
// by known answers from the Python `blake3` module (tests/golden/blake3_kat.json).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

namespace b3 {

static const uint32_t kIV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t kPerm[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };

static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
static inline void g(uint32_t* s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
  s[a] = s[a] + s[b] + mx; s[d] = rotr(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];      s[b] = rotr(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + my; s[d] = rotr(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];      s[b] = rotr(s[b] ^ s[c], 7);
}
// Full 16-word compression output.
static inline void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter,
                            uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    kIV[0], kIV[1], kIV[2], kIV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                    block_len, flags};
  uint32_t m[16];
  std::memcpy(m, block, 64);
  for (int r = 0; r < 7; ++r) {
    g(s, 0, 4, 8, 12, m[0], m[1]);   g(s, 1, 5, 9, 13, m[2], m[3]);
    g(s, 2, 6, 10, 14, m[4], m[5]);  g(s, 3, 7, 11, 15, m[6], m[7]);
    g(s, 0, 5, 10, 15, m[8], m[9]);  g(s, 1, 6, 11, 12, m[10], m[11]);
    g(s, 2, 7, 8, 13, m[12], m[13]); g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; ++i) t[i] = m[kPerm[i]];
      std::memcpy(m, t, 64);
    }
  }
  for (int i = 0; i < 8; ++i) { out[i] = s[i] ^ s[i + 8]; out[i + 8] = s[i + 8] ^ cv[i]; }
}
static inline void words_from_bytes(const uint8_t* p, size_t n, uint32_t w[16]) {
  uint8_t buf[64] = {0};
  std::memcpy(buf, p, n);
  for (int i = 0; i < 16; ++i)
    w[i] = (uint32_t)buf[4 * i] | ((uint32_t)buf[4 * i + 1] << 8) |
           ((uint32_t)buf[4 * i + 2] << 16) | ((uint32_t)buf[4 * i + 3] << 24);
}

// Streaming hasher: update() any number of times, then finalize().
struct Hasher {
  uint32_t cv[8];             // current chunk's chaining value
  uint64_t chunk_counter = 0;
  uint8_t block[64];
  uint32_t block_len = 0;
  uint32_t blocks_compressed = 0;
  uint32_t stack[54][8];       // chaining values of completed subtrees
  int stack_len = 0;

  Hasher() { std::memcpy(cv, kIV, 32); }

  uint32_t start_flag() const { return blocks_compressed == 0 ? CHUNK_START : 0; }
  size_t chunk_len() const { return 64 * (size_t)blocks_compressed + block_len; }

  void parent_cv(const uint32_t l[8], const uint32_t r[8], uint32_t out[8]) {
    uint32_t blk[16], o[16];
    std::memcpy(blk, l, 32); std::memcpy(blk + 8, r, 32);
    compress(kIV, blk, 0, 64, PARENT, o);
    std::memcpy(out, o, 32);
  }
  void add_chunk_cv(uint32_t ncv[8], uint64_t total_chunks) {
    while ((total_chunks & 1) == 0) {
      parent_cv(stack[--stack_len], ncv, ncv);
      total_chunks >>= 1;
    }
    std::memcpy(stack[stack_len++], ncv, 32);
  }
  void update(const void* data, size_t n) {
    const uint8_t* p = (const uint8_t*)data;
    while (n > 0) {
      if (chunk_len() == 1024) {  // finish the full chunk: more input follows
        uint32_t w[16], o[16];
        words_from_bytes(block, block_len, w);
        compress(cv, w, chunk_counter, block_len, start_flag() | CHUNK_END, o);
        uint32_t ccv[8];
        std::memcpy(ccv, o, 32);
        uint64_t total = chunk_counter + 1;
        add_chunk_cv(ccv, total);
        std::memcpy(cv, kIV, 32);
        chunk_counter = total;
        block_len = 0;
        blocks_compressed = 0;
      }
      if (block_len == 64) {  // a full block with more input after it
        uint32_t w[16], o[16];
        words_from_bytes(block, 64, w);
        compress(cv, w, chunk_counter, 64, start_flag(), o);
        std::memcpy(cv, o, 32);
        blocks_compressed++;
        block_len = 0;
      }
      size_t want = 1024 - chunk_len();
      size_t room = 64 - block_len;
      size_t take = n < room ? n : room;
      if (take > want) take = want;
      std::memcpy(block + block_len, p, take);
      block_len += (uint32_t)take;
      p += take;
      n -= take;
    }
  }
  void finalize(uint8_t out32[32]) {
    // Output node: the current chunk's last block, then parents up the stack.
    uint32_t in_cv[8], blk[16];
    uint64_t counter = chunk_counter;
    uint32_t blen = block_len;
    uint32_t flags = start_flag() | CHUNK_END;
    std::memcpy(in_cv, cv, 32);
    words_from_bytes(block, block_len, blk);
    int i = stack_len;
    while (i > 0) {
      uint32_t o[16];
      compress(in_cv, blk, counter, blen, flags, o);
      uint32_t right[8];
      std::memcpy(right, o, 32);
      --i;
      std::memcpy(blk, stack[i], 32);
      std::memcpy(blk + 8, right, 32);
      std::memcpy(in_cv, kIV, 32);
      counter = 0; blen = 64; flags = PARENT;
    }
    uint32_t o[16];
    compress(in_cv, blk, counter, blen, flags | ROOT, o);
    for (int k = 0; k < 8; ++k) {
      out32[4 * k] = (uint8_t)o[k]; out32[4 * k + 1] = (uint8_t)(o[k] >> 8);
      out32[4 * k + 2] = (uint8_t)(o[k] >> 16); out32[4 * k + 3] = (uint8_t)(o[k] >> 24);
    }
  }
  void update_u8(uint8_t v) { update(&v, 1); }
  void update_u32(uint32_t v) { uint8_t b[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)}; update(b, 4); }
  void update_u64(uint64_t v) { update_u32((uint32_t)v); update_u32((uint32_t)(v >> 32)); }
};

}  // namespace b3
