// Basis-state kernels: prefix scans, key packing, the basis hash, Cmax, heat-bath candidate
// generation with warp-free load balancing, candidate compaction and an LSD radix sort of packed
// keys.  All are memory-bound integer/byte kernels sized in grid-stride loops.
#include <atomic>

#include "ops.h"

namespace vhci {

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int64_t kScanTile = kScanThreads * kScanItems;  // 4096

inline int grid_for(int64_t n, int threads, int max_blocks = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix, total in *tot.
__device__ int64_t block_excl_scan(int64_t v, int64_t* warp_sums, int64_t* tot) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int64_t s = lane < nw ? warp_sums[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  const int64_t base = wid ? warp_sums[wid - 1] : 0;
  *tot = warp_sums[nw - 1];
  __syncthreads();
  return base + incl - v;
}

template <typename TI>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const TI* __restrict__ in, int64_t n,
                                                              int64_t* __restrict__ bsum) {
  __shared__ int64_t ws[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t s = 0;
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
    if (i < n) s += (int64_t)in[i];
  }
  int64_t tot;
  block_excl_scan(s, ws, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// Exclusive scan of one tile, adding `offs[blockIdx.x]` (or 0); the last block writes out[n].
template <typename TI>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const TI* __restrict__ in, int64_t* out,
                                                            int64_t n, const int64_t* offs) {
  __shared__ int64_t sm[kScanTile];
  __shared__ int64_t ws[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
    sm[j * kScanThreads + threadIdx.x] = i < n ? (int64_t)in[i] : 0;
  }
  __syncthreads();
  int64_t loc[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) { loc[j] = sm[threadIdx.x * kScanItems + j]; s += loc[j]; }
  int64_t tot;
  int64_t pre = block_excl_scan(s, ws, &tot);
  const int64_t off = offs ? offs[blockIdx.x] : 0;
  pre += off;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    sm[threadIdx.x * kScanItems + j] = pre;
    pre += loc[j];
  }
  __syncthreads();
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + (int64_t)j * kScanThreads + threadIdx.x;
    if (i < n) out[i] = sm[j * kScanThreads + threadIdx.x];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + tot;
}

template <typename TI>
void scan_impl(const TI* in, int64_t* out, int64_t n, int64_t* tmp, cudaStream_t s) {
  if (n <= kScanTile) {
    note_launch(); k_scan_tile<TI><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
    return;
  }
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  note_launch(); k_scan_reduce<TI><<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, tmp);
  scan_impl<int64_t>(tmp, tmp, nb, tmp + nb + 1, s);
  note_launch(); k_scan_tile<TI><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, tmp);
}

}  // namespace

int64_t scan_tmp_elems(int64_t n) {
  if (n <= kScanTile) return 0;
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  return nb + 1 + scan_tmp_elems(nb);
}

void exclusive_scan(const int64_t* in, int64_t* out, int64_t n, int64_t* tmp, cudaStream_t s) {
  scan_impl<int64_t>(in, out, n, tmp, s);
}
void exclusive_scan_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* tmp,
                        cudaStream_t s) {
  scan_impl<int32_t>(in, out, n, tmp, s);
}

// ---------------------------------------------------------------- keys and the basis hash ----

namespace {

__global__ void k_pack(const uint8_t* __restrict__ q, int64_t n, int nm, KeyLayout L,
                       uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int w = 0; w < L.W; ++w) {
      uint64_t v = 0;
      for (int j = 0; j < L.mpw; ++j) {
        const int m = w * L.mpw + j;
        if (m < nm) v |= (uint64_t)q[i * nm + m] << (j * L.bits);
      }
      keys[i * L.W + w] = v;
    }
  }
}

__global__ void k_unpack(const uint64_t* __restrict__ keys, int64_t n, int nm, KeyLayout L,
                         uint8_t* __restrict__ q) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int m = 0; m < nm; ++m) {
      const uint64_t v = keys[i * L.W + m / L.mpw];
      q[i * nm + m] = (uint8_t)((v >> ((m % L.mpw) * L.bits)) & ((1u << L.bits) - 1u));
    }
}

__global__ void k_repack(const uint64_t* __restrict__ in, KeyLayout A, uint64_t* __restrict__ out,
                         KeyLayout B, int64_t n, int nm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int w = 0; w < B.W; ++w) {
      uint64_t v = 0;
      for (int j = 0; j < B.mpw; ++j) {
        const int m = w * B.mpw + j;
        if (m >= nm) break;
        const uint64_t a = in[i * A.W + m / A.mpw];
        const uint64_t q = (a >> ((m % A.mpw) * A.bits)) & ((1u << A.bits) - 1u);
        v |= q << (j * B.bits);
      }
      out[i * B.W + w] = v;
    }
  }
}

__global__ void k_fill_u64(uint64_t* p, uint64_t n, uint64_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

template <int W>
__global__ void k_hash_insert(uint64_t* slots, uint64_t mask, const uint64_t* __restrict__ keys,
                              int64_t begin, int64_t end, int* flags) {
  for (int64_t i = begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k[W];
    load_key<W>(keys, i, k);
    hash_insert_unique<W>(slots, mask, keys, k, key_hash<W>(k), (uint32_t)i, flags);
  }
}

template <int W>
void hash_insert_launch(uint64_t* slots, uint64_t mask, const uint64_t* keys, int64_t begin,
                        int64_t end, int* flags, cudaStream_t s) {
  if (end <= begin) return;
  note_launch(); k_hash_insert<W><<<grid_for(end - begin, 256), 256, 0, s>>>(slots, mask, keys, begin, end,
                                                               flags);
}

__global__ void k_max_quanta(const uint64_t* __restrict__ keys, int64_t n, int nm, KeyLayout L,
                             int* out) {
  __shared__ int sm[256];
  for (int m = threadIdx.x; m < nm; m += blockDim.x) sm[m] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int m = 0; m < nm; ++m) {
      const int q = (int)((keys[i * L.W + m / L.mpw] >> ((m % L.mpw) * L.bits)) &
                          ((1u << L.bits) - 1u));
      if (q > sm[m]) atomicMax(sm + m, q);
    }
  __syncthreads();
  for (int m = threadIdx.x; m < nm; m += blockDim.x) atomicMax(out + m, sm[m]);
}

}  // namespace

void pack_keys(const uint8_t* q, int64_t n, int nm, KeyLayout L, uint64_t* keys, cudaStream_t s) {
  if (n > 0) { note_launch(); k_pack<<<grid_for(n, 256), 256, 0, s>>>(q, n, nm, L, keys); }
}
void unpack_keys(const uint64_t* keys, int64_t n, int nm, KeyLayout L, uint8_t* q,
                 cudaStream_t s) {
  if (n > 0) { note_launch(); k_unpack<<<grid_for(n, 256), 256, 0, s>>>(keys, n, nm, L, q); }
}
void repack_keys(const uint64_t* in, KeyLayout A, uint64_t* out, KeyLayout B, int64_t n, int nm,
                 cudaStream_t s) {
  if (n > 0) { note_launch(); k_repack<<<grid_for(n, 256), 256, 0, s>>>(in, A, out, B, n, nm); }
}
void hash_clear(uint64_t* slots, uint64_t nslots, cudaStream_t s) {
  note_launch(); k_fill_u64<<<grid_for((int64_t)nslots, 256), 256, 0, s>>>(slots, nslots, kEmptySlot);
}
void hash_insert_range(uint64_t* slots, uint64_t mask, const uint64_t* keys, int64_t begin,
                       int64_t end, int W, int* flags, cudaStream_t s) {
  VHCI_DISPATCH_W(W, hash_insert_launch, slots, mask, keys, begin, end, flags, s);
}
void max_quanta_per_mode(const uint64_t* keys, int64_t n, int nm, KeyLayout L, int* out,
                         cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(int) * nm, s);
  if (n > 0) { note_launch(); k_max_quanta<<<grid_for(n, 256, 592), 256, 0, s>>>(keys, n, nm, L, out); }
}

// ------------------------------------------------------------------------- heat-bath selection

namespace {

// One warp per row: signed entry of largest |C_ij| over j < nopt, lowest j on ties
// (HB.cpp:204-214: strict '>' keeps the first occurrence).
__global__ void k_cmax(const double* __restrict__ X, int64_t n, int ldx, int nopt,
                       double* __restrict__ cmax) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    double best = -1.0;
    int bj = 0x7fffffff;
    for (int j = lane; j < nopt; j += 32) {
      const double a = fabs(X[i * ldx + j]);
      if (a > best) { best = a; bj = j; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oj = __shfl_xor_sync(0xffffffffu, bj, o);
      if (ob > best || (ob == best && oj < bj)) { best = ob; bj = oj; }
    }
    if (lane == 0) cmax[i] = (bj < nopt) ? X[i * ldx + bj] : 0.0;
  }
}

// Pattern count of state i: the heat-bath list is sorted by |fc| descending, so the FCs with
// fl(|C_i| * |fc|) >= eps form a prefix (the reference's `break`, HB.cpp:26,172); its length is
// found by binary search and mapped to a pattern count through the prefix table.
__global__ void k_select_count(const double* __restrict__ cmax, int64_t n, HBTable hb, double eps,
                               int64_t* __restrict__ work) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double c = fabs(cmax[i]);
    int lo = 0, hi = hb.nhb;  // first f failing the test
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (c * __ldg(hb.absfc + mid) >= eps) lo = mid + 1; else hi = mid;
    }
    work[i] = __ldg(hb.cum + lo);
  }
}

// Work item w -> (state, FC, pattern) -> candidate key.  Consecutive items share state and FC,
// so warps stay converged; the basis hash is L2-resident for every workload here.
template <int W>
__global__ void __launch_bounds__(256) k_select_gen(const uint64_t* __restrict__ keys, int64_t n,
                                                    const int64_t* __restrict__ woff,
                                                    int64_t total, HBTable hb, KeyLayout L,
                                                    HashView basis, NewSetView ns) {
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < total;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = upper_index(woff, n, w);
    const int64_t r = w - __ldg(woff + i);
    const int f = (int)upper_index(hb.cum, hb.nhb, r);
    int t = (int)(r - __ldg(hb.cum + f));
    const HBDev e = hb.e[f];
    if (e.zero_idx >= 0 && t >= e.zero_idx) ++t;
    uint64_t k[W];
    load_key<W>(keys, i, k);
    bool ok = true, over = false;
    for (int j = e.nk - 1; j >= 0; --j) {
      const int base = e.pw[j] + 1;
      const int d = 2 * (t % base) - e.pw[j];
      t /= base;
      const int q = key_q<W>(k, e.mode[j], L.mpw, L.bits) + d;
      if (q < 0) { ok = false; break; }
      if (q > L.qmax) { over = true; continue; }
      key_add<W>(k, e.mode[j], L.mpw, L.bits, d);
    }
    if (!ok) continue;
    if (over) { atomicOr(ns.flags, kFlagKeyOverflow); continue; }
    const uint64_t h = key_hash<W>(k);
    if (hash_find<W>(basis, k, h) >= 0) continue;
    newset_insert<W>(ns, k, h);
  }
}

template <int W>
void select_gen_launch(const uint64_t* keys, int64_t n, const int64_t* woff, int64_t total,
                       HBTable hb, KeyLayout L, HashView basis, NewSetView ns, cudaStream_t s) {
  if (total <= 0) return;
  note_launch(); k_select_gen<W><<<grid_for(total, 256, 148 * 32), 256, 0, s>>>(keys, n, woff, total, hb, L,
                                                                basis, ns);
}

__global__ void k_compact(const uint64_t* __restrict__ cand, const uint8_t* __restrict__ dead,
                          int64_t ncand, int W, uint64_t* __restrict__ out,
                          unsigned long long* n_out) {
  const int lane = threadIdx.x & 31;
  for (int64_t c0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) & ~31ll; c0 < ncand;
       c0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = c0 + lane;
    const bool live = c < ncand && !dead[c];
    const unsigned b = __ballot_sync(0xffffffffu, live);
    unsigned long long base = 0;
    if (lane == 0 && b) base = atomicAdd(n_out, (unsigned long long)__popc(b));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (live) {
      const unsigned long long pos = base + __popc(b & lanemask_lt());
      for (int w = 0; w < W; ++w) out[pos * W + w] = cand[c * W + w];
    }
  }
}

}  // namespace

void cmax_rows(const double* X, int64_t n, int ldx, int nopt, double* cmax, cudaStream_t s) {
  if (n > 0) { note_launch(); k_cmax<<<grid_for(n * 32, 256), 256, 0, s>>>(X, n, ldx, nopt, cmax); }
}
void select_count(const double* cmax, int64_t n, HBTable hb, double eps, int64_t* work,
                  cudaStream_t s) {
  if (n > 0) { note_launch(); k_select_count<<<grid_for(n, 256), 256, 0, s>>>(cmax, n, hb, eps, work); }
}
void select_generate(const uint64_t* keys, int64_t n, const int64_t* woff, int64_t total,
                     HBTable hb, KeyLayout L, HashView basis, NewSetView ns, cudaStream_t s) {
  VHCI_DISPATCH_W(L.W, select_gen_launch, keys, n, woff, total, hb, L, basis, ns, s);
}
void newset_compact(const uint64_t* cand, const uint8_t* dead, int64_t ncand, int W,
                    uint64_t* out, unsigned long long* n_out, cudaStream_t s) {
  cudaMemsetAsync(n_out, 0, sizeof(unsigned long long), s);
  if (ncand > 0) {
    note_launch();
    k_compact<<<grid_for(ncand, 256), 256, 0, s>>>(cand, dead, ncand, W, out, n_out);
  }
}

// ------------------------------------------------------------------------------- radix sort ---

namespace {

constexpr int kRadixThreads = 256;
constexpr int kRadixRounds = 16;
constexpr int64_t kRadixTile = kRadixThreads * kRadixRounds;  // 4096 keys per block

template <int W>
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint64_t* __restrict__ keys,
                                                              int64_t n, int word, int shift,
                                                              int64_t* __restrict__ hist,
                                                              int nblk) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    const int64_t i = base + r * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(h + ((keys[i * W + word] >> shift) & 255u), 1);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: within a round of 256 keys (one per thread, in thread order) a key's rank is
// (same-digit keys in earlier warps) + (same-digit keys in earlier lanes of its warp); rounds are
// processed in order and blocks receive their digit offsets from the global scan.
template <int W>
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(
    const uint64_t* __restrict__ keys, uint64_t* __restrict__ out, int64_t n, int word, int shift,
    const int64_t* __restrict__ offs, int nblk) {
  __shared__ int wc[kRadixThreads / 32][256];
  __shared__ int64_t run[256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  run[threadIdx.x] = offs[(int64_t)threadIdx.x * nblk + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    for (int w = 0; w < kRadixThreads / 32; ++w) wc[w][threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = base + r * kRadixThreads + threadIdx.x;
    const bool valid = i < n;
    uint64_t k[W];
    int d = 256 + lane;  // unique non-digit for invalid lanes
    if (valid) {
      load_key<W>(keys, i, k);
      d = (int)((k[word] >> shift) & 255u);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lanemask_lt());
    if (valid && rank == 0) wc[wid][d] = __popc(peers);
    __syncthreads();
    {
      int acc = 0;
      const int dg = threadIdx.x;
      for (int w = 0; w < kRadixThreads / 32; ++w) {
        const int c = wc[w][dg];
        wc[w][dg] = acc;
        acc += c;
      }
      __syncthreads();
      if (valid) {
        const int64_t pos = run[d] + wc[wid][d] + rank;
#pragma unroll
        for (int w = 0; w < W; ++w) out[pos * W + w] = k[w];
      }
      __syncthreads();
      run[dg] += acc;
    }
    __syncthreads();
  }
}

template <int W>
void radix_launch(uint64_t* keys, uint64_t* alt, int64_t n, int nbits, int64_t* hist,
                  cudaStream_t s) {
  const int nblk = (int)((n + kRadixTile - 1) / kRadixTile);
  const int64_t hn = (int64_t)256 * nblk;
  int64_t* offs = hist;
  int64_t* tmp = hist + hn + 1;
  uint64_t* src = keys;
  uint64_t* dst = alt;
  int passes = 0;
  for (int b = 0; b < nbits; b += 8) {
    const int word = b / 64, shift = b % 64;
    note_launch(); k_radix_hist<W><<<nblk, kRadixThreads, 0, s>>>(src, n, word, shift, offs, nblk);
    exclusive_scan(offs, offs, hn, tmp, s);
    note_launch(); k_radix_scatter<W><<<nblk, kRadixThreads, 0, s>>>(src, dst, n, word, shift, offs, nblk);
    uint64_t* t = src; src = dst; dst = t;
    ++passes;
  }
  if (passes & 1) cudaMemcpyAsync(keys, src, sizeof(uint64_t) * n * W, cudaMemcpyDeviceToDevice, s);
}

}  // namespace

int64_t radix_hist_elems(int64_t n) {
  const int64_t nblk = (n + kRadixTile - 1) / kRadixTile;
  const int64_t hn = 256 * nblk;
  return hn + 1 + scan_tmp_elems(hn);
}

void radix_sort_keys(uint64_t* keys, uint64_t* alt, int64_t n, int W, int nbits, int64_t* hist,
                     cudaStream_t s) {
  if (n <= 1) return;
  VHCI_DISPATCH_W(W, radix_launch, keys, alt, n, nbits, hist, s);
}

}  // namespace vhci
