// Device-side building blocks: packed basis-state keys, hashing, the open-addressing tables and
// small warp utilities.  All kernels are written for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace vhci {

// Error flags raised by kernels (bit mask in a device word read back by the host).
enum : int {
  kFlagKeyOverflow = 1,   // a generated state needs more quanta per mode than the key layout holds
  kFlagTableFull = 2,     // a probe sequence exceeded its bound
  kFlagCandOverflow = 4,  // candidate buffer too small
  kFlagDuplicate = 8,     // a key inserted twice into a unique-key table
};

constexpr uint64_t kEmptySlot = ~0ull;
constexpr uint32_t kNoIndex = 0xFFFFFFFFu;

// Packed key layout: `bits` (4 or 8) per mode, 64/bits modes per 64-bit word, W words per state.
// Mode m lives in word m / mpw at bit offset (m % mpw) * bits.  Unused high fields are zero.
struct KeyLayout {
  int bits;   // 4 or 8
  int mpw;    // modes per word
  int W;      // words per key
  int qmax;   // largest storable quanta (15 or 255)
};

__host__ __device__ inline int key_word(int m, int mpw) { return m / mpw; }
__host__ __device__ inline int key_shift(int m, int mpw, int bits) { return (m % mpw) * bits; }

// Quanta of mode m from a key held in registers (W words); the word is picked without dynamic
// register indexing.
template <int W>
__device__ __forceinline__ int key_q(const uint64_t (&k)[W], int m, int mpw, int bits) {
  const int w = m / mpw;
  uint64_t v = k[0];
#pragma unroll
  for (int i = 1; i < W; ++i)
    if (w == i) v = k[i];
  return (int)((v >> ((m % mpw) * bits)) & ((1u << bits) - 1u));
}

template <int W>
__device__ __forceinline__ void key_add(uint64_t (&k)[W], int m, int mpw, int bits, int d) {
  const int w = m / mpw;
  const uint64_t add = (uint64_t)((int64_t)d << ((m % mpw) * bits));
#pragma unroll
  for (int i = 0; i < W; ++i)
    if (w == i) k[i] += add;
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

template <int W>
__device__ __forceinline__ uint64_t key_hash(const uint64_t (&k)[W]) {
  uint64_t h = mix64(k[0] ^ 0x9E3779B97F4A7C15ull);
#pragma unroll
  for (int i = 1; i < W; ++i) h = mix64(h ^ (k[i] + 0x632BE59BD9B4E019ull * (uint64_t)i));
  return h;
}

template <int W>
__device__ __forceinline__ void load_key(const uint64_t* __restrict__ keys, int64_t i,
                                         uint64_t (&k)[W]) {
#pragma unroll
  for (int w = 0; w < W; ++w) k[w] = keys[i * W + w];
}

template <int W>
__device__ __forceinline__ bool key_eq(const uint64_t* __restrict__ keys, int64_t i,
                                       const uint64_t (&k)[W]) {
  bool eq = true;
#pragma unroll
  for (int w = 0; w < W; ++w) eq &= (keys[i * W + w] == k[w]);
  return eq;
}

// Read-only view of a unique-key hash: slot = (fingerprint << 32) | index into `keys`.
struct HashView {
  const uint64_t* __restrict__ slots;
  uint64_t mask;
  const uint64_t* __restrict__ keys;
};

// Returns the key's index or -1.  Linear probing; at load <= 1/2 a miss ends after ~2.5 slots.
template <int W>
__device__ __forceinline__ int64_t hash_find(const HashView& t, const uint64_t (&k)[W],
                                             uint64_t h) {
  uint64_t s = h & t.mask;
  const uint32_t fp = (uint32_t)(h >> 32);
  for (uint64_t it = 0; it <= t.mask; ++it) {
    const uint64_t v = __ldg(t.slots + s);
    if (v == kEmptySlot) return -1;
    if ((uint32_t)(v >> 32) == fp) {
      const uint32_t idx = (uint32_t)v;
      if (key_eq<W>(t.keys, idx, k)) return idx;
    }
    s = (s + 1) & t.mask;
  }
  return -1;
}

// Insert a key known to be absent (basis keys are unique).  Bounded by the table size.
template <int W>
__device__ __forceinline__ void hash_insert_unique(uint64_t* slots, uint64_t mask,
                                                   const uint64_t* keys, const uint64_t (&k)[W],
                                                   uint64_t h, uint32_t idx, int* flags) {
  uint64_t s = h & mask;
  const uint64_t val = ((uint64_t)(uint32_t)(h >> 32) << 32) | idx;
  for (uint64_t it = 0; it <= mask; ++it) {
    const uint64_t old = atomicCAS((unsigned long long*)(slots + s), kEmptySlot, val);
    if (old == kEmptySlot) return;
    if ((old >> 32) == (val >> 32) && key_eq<W>(keys, (uint32_t)old, k)) {
      atomicOr(flags, kFlagDuplicate);
      return;
    }
    s = (s + 1) & mask;
  }
  atomicOr(flags, kFlagTableFull);
}

// Concurrent insert-if-absent set whose keys live in a candidate buffer.  A thread that finds an
// empty slot first writes its key to a fresh candidate entry, fences, then publishes it by CAS; a
// thread that meets an equal key marks its own candidate (if any) dead.  The set is the live
// candidates.  Bounded by `max_probe`; overflow of either bound raises a flag.
struct NewSetView {
  uint64_t* slots;
  uint64_t mask;
  uint64_t* cand;          // candidate keys, W words each
  uint8_t* dead;           // 1 = duplicate candidate
  unsigned long long* count;
  uint64_t cap;            // candidate capacity
  int* flags;
};

template <int W>
__device__ __forceinline__ void newset_insert(const NewSetView& ns, const uint64_t (&k)[W],
                                              uint64_t h) {
  uint64_t s = h & ns.mask;
  const uint32_t fp = (uint32_t)(h >> 32);
  unsigned long long mine = ~0ull;
  for (uint64_t it = 0; it <= ns.mask; ++it) {
    uint64_t v = *(volatile uint64_t*)(ns.slots + s);
    if (v == kEmptySlot) {
      if (mine == ~0ull) {
        mine = atomicAdd(ns.count, 1ull);
        if (mine >= ns.cap) {
          atomicOr(ns.flags, kFlagCandOverflow);
          return;
        }
#pragma unroll
        for (int w = 0; w < W; ++w) __stcg(ns.cand + mine * W + w, k[w]);
        __threadfence();
      }
      const uint64_t val = ((uint64_t)fp << 32) | (uint32_t)mine;
      const uint64_t old = atomicCAS((unsigned long long*)(ns.slots + s), kEmptySlot, val);
      if (old == kEmptySlot) return;
      v = old;
    }
    if ((uint32_t)(v >> 32) == fp) {
      __threadfence();
      const uint32_t idx = (uint32_t)v;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= (__ldcg(ns.cand + (uint64_t)idx * W + w) == k[w]);
      if (eq) {
        if (mine != ~0ull) ns.dead[mine] = 1;
        return;
      }
    }
    s = (s + 1) & ns.mask;
  }
  atomicOr(ns.flags, kFlagTableFull);
  if (mine != ~0ull) ns.dead[mine] = 1;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Largest index i in [0, n) with a[i] <= x (a non-decreasing, a[0] <= x).
__device__ __forceinline__ int64_t upper_index(const int64_t* __restrict__ a, int64_t n,
                                               int64_t x) {
  int64_t lo = 0, hi = n;  // invariant: a[lo] <= x, answer in [lo, hi)
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= x) lo = mid; else hi = mid;
  }
  return lo;
}

}  // namespace vhci

#define VHCI_DISPATCH_W(W_RUNTIME, FN, ...)                   \
  switch (W_RUNTIME) {                                       \
    case 1: FN<1>(__VA_ARGS__); break;                        \
    case 2: FN<2>(__VA_ARGS__); break;                        \
    case 3: FN<3>(__VA_ARGS__); break;                        \
    case 4: FN<4>(__VA_ARGS__); break;                        \
    case 5: FN<5>(__VA_ARGS__); break;                        \
    case 6: FN<6>(__VA_ARGS__); break;                        \
    case 7: FN<7>(__VA_ARGS__); break;                        \
    case 8: FN<8>(__VA_ARGS__); break;                        \
    default: break;                                          \
  }
