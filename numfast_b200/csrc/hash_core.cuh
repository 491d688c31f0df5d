// Global open-addressing table of int32 keys (slot word = 1 << 32 | key,
// 0 = empty; linear probing from a multiplicative hash).  Shared by the
// HASH and SHARED_HASH strategies.
#pragma once

#include "groupby_core.cuh"

namespace nfc {

NFC_DEV uint64_t key_hash64(int32_t key) { return (uint64_t)(uint32_t)key * 0x9E3779B97F4A7C15ull; }

// Slot of `key`, inserting it if absent, after at most `limit` probes;
// -1 when none was free.
NFC_DEV int64_t hash_slot_bounded(uint64_t* table, int lg, int32_t key, uint64_t limit) {
  const uint64_t w = (1ull << 32) | (uint32_t)key;
  const uint64_t mask = (1ull << lg) - 1;
  const uint64_t h = key_hash64(key) >> (64 - lg);
  if (limit > mask + 1) limit = mask + 1;
  for (uint64_t i = 0; i < limit; ++i) {
    const uint64_t slot = (h + i) & mask;
    uint64_t cur = table[slot];
    if (cur == w) return (int64_t)slot;
    if (cur == 0) {
      cur = atomicCAS(reinterpret_cast<unsigned long long*>(table) + slot, 0ull, (unsigned long long)w);
      if (cur == 0 || cur == w) return (int64_t)slot;
    }
  }
  return -1;
}

// Full-length probe; a full table records NFC_ERR_RANGE.
NFC_DEV int64_t hash_slot(uint64_t* table, int lg, int32_t key, int32_t* err) {
  const int64_t s = hash_slot_bounded(table, lg, key, ~0ull);
  if (s < 0) atomicExch(err, NFC_ERR_RANGE);
  return s;
}

}  // namespace nfc
