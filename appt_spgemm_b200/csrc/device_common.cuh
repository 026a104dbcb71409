// Device helpers shared by the engine's kernels: lane groups, shared-memory
// hashing, bitonic sorting and block-level scans.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace spg {

// A matrix as the kernels see it (B is A, or the engine's transpose of A).
struct MatView {
  int32_t n;
  int64_t nnz;
  const int32_t* __restrict__ rowptr;
  const int32_t* __restrict__ col;
  const double* __restrict__ val;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ void report(uint32_t* status, uint32_t bits) {
  atomicOr(status, bits);
}

// Multiply-shift hash: the high bits of j·φ·2^32 select one of 2^LOG2T slots.
// (The reference keeps the low bits of j·2654435761, src/spgemm_engine.cuh:64,
// so keys congruent modulo the table size collide; the high bits do not.)
template <int LOG2T>
__device__ __forceinline__ unsigned hash_slot(int j) {
  return ((unsigned)j * 0x9E3779B1u) >> (32 - LOG2T);
}

// CAS-first linear probe of the hash-table kernels: one shared atomic per probe, the
// loop exits on an empty slot (claimed) or on the key itself (reading the slot
// first and claiming only empty ones measured slower: 3.32 vs 2.88 ms for the
// numeric phase of the 96³ stencil; so did claims without atomics — a round of
// read, __match_any_sync grouping of the lanes that saw an empty slot, write by
// each group's lowest lane and two __syncwarp per round — 4.48 vs 2.83 ms per
// numeric launch and 2.25 vs 1.07 ms per symbolic one; and so did skipping the
// CAS for the lanes whose column the previous segment already inserted, found
// by a five-step shuffle search over that segment's columns — 8.26 vs 5.67 ms
// per step numeric, 4.32 vs 2.14 symbolic: the shuffles share this kernel's
// saturated shared-memory pipe).  In the numeric phase the value is then
// 0.0 + v for a freshly claimed slot and slot + v otherwise, so no value array
// is cleared between rows.
template <int LOG2T, bool NUMERIC>
__device__ __forceinline__ void insert_acc(int* keys, double* vals, int j, double v,
                                           uint32_t* status) {
  constexpr unsigned T = 1u << LOG2T;
  unsigned h = hash_slot<LOG2T>(j);
  int old = atomicCAS(keys + h, kEmptyKey, j);
  unsigned probe = 1;
  while (old != kEmptyKey && old != j) {
    if (probe++ == T) {
      report(status, DEV_ERR_HASH_FULL);
      return;
    }
    h = (h + 1) & (T - 1);
    old = atomicCAS(keys + h, kEmptyKey, j);
  }
  if (NUMERIC) {
    // a freshly claimed slot starts from 0.0 without reading the stale value
    double cur = 0.0;
    if (old != kEmptyKey) cur = vals[h];
    vals[h] = __dadd_rn(cur, v);
  }
}

// ---- lane groups -------------------------------------------------------------
// A row is processed by a group of G lanes: a power-of-two slice of one warp
// (G <= 32, several rows per CTA) or the whole CTA (G = blockDim.x > 32).
struct WarpGroup {
  int G;        // lanes in the group (power of two, <= 32)
  int lane;     // 0..G-1
  int base;     // first lane of the group within its warp
  unsigned mask;
  __device__ __forceinline__ WarpGroup(int g) : G(g) {
    int wl = threadIdx.x & 31;
    lane = wl & (g - 1);
    base = wl & ~(g - 1);
    mask = (g == 32) ? 0xffffffffu : (((1u << g) - 1u) << base);
  }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ unsigned ballot(bool p) const {
    return (__ballot_sync(mask, p) & mask) >> base;
  }
  __device__ __forceinline__ int sum(int v) const {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, 32);
    return v;
  }
  __device__ __forceinline__ long long sum64(long long v) const {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, 32);
    return v;
  }
};

struct CtaGroup {
  int G;
  int lane;
  __device__ __forceinline__ CtaGroup() : G(blockDim.x), lane(threadIdx.x) {}
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Block-wide sum of an int (all threads return the total).  `scratch` holds
// 32 ints; the call contains two __syncthreads.
__device__ __forceinline__ long long block_sum64(long long v, long long* scratch) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) scratch[w] = v;
  __syncthreads();
  long long t = 0;
  for (int i = 0; i < nw; ++i) t += scratch[i];
  return t;
}

// The CTA's next work item: one thread draws it from a counter that the
// launcher zeroed; every thread of the CTA returns the same index.
__device__ __forceinline__ int next_cta_item(int32_t* counter, int* s_next) {
  __syncthreads();  // every thread has read the previous item
  if (threadIdx.x == 0) *s_next = atomicAdd(counter, 1);
  __syncthreads();
  return *s_next;
}

// The CTA's it-th work item of nitems.  A persistent launch (fewer CTAs than
// items) draws items from the counter as CTAs free up, so costly items do not
// pile up on a few CTAs.  A launch of a CTA per item takes item blockIdx.x and
// retires after it: the hardware hands out the CTAs as SMs free up, and work
// on a higher-priority stream gets the SMs in between (a CTA that kept drawing
// would hold its SM until the last item).  Items past the end come back as
// nitems.
__device__ __forceinline__ int cta_item(int32_t* counter, int nitems, int it, int* s_next) {
  if (counter && (int)gridDim.x < nitems) return next_cta_item(counter, s_next);
  const long long r = (long long)blockIdx.x + (long long)it * gridDim.x;
  return r < nitems ? (int)r : nitems;
}

// Block-wide exclusive scan of an int; returns this thread's prefix and sets
// *total.  `scratch` holds 33 ints.  Contains two __syncthreads.
__device__ __forceinline__ int block_exclusive_scan(int v, int* scratch, int* total) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  int incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();
  if (lane == 31) scratch[w] = incl;
  __syncthreads();
  int before = 0, all = 0;
  for (int i = 0; i < nw; ++i) {
    int s = scratch[i];
    if (i < w) before += s;
    all += s;
  }
  *total = all;
  return before + incl - v;
}

// ---- bitonic sort of (key, value) pairs in shared memory ---------------------
// Sorts keys[0..P) ascending (P a power of two) carrying vals along, by the G
// lanes of a group.  Ties cannot occur for the engine's unique keys; padding
// keys are INT_MAX.
template <class Grp>
__device__ __forceinline__ void bitonic_sort_pairs(const Grp& g, int* keys, double* vals, int P) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = g.lane; i < (P >> 1); i += g.G) {
        int lo = ((i & ~(jj - 1)) << 1) | (i & (jj - 1));
        int hi = lo + jj;
        bool asc = (lo & k) == 0;
        int klo = keys[lo], khi = keys[hi];
        if ((klo > khi) == asc) {
          keys[lo] = khi;
          keys[hi] = klo;
          double t = vals[lo];
          vals[lo] = vals[hi];
          vals[hi] = t;
        }
      }
      g.sync();
    }
  }
}

template <class Grp>
__device__ __forceinline__ void bitonic_sort_keys(const Grp& g, int* keys, int P) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = g.lane; i < (P >> 1); i += g.G) {
        int lo = ((i & ~(jj - 1)) << 1) | (i & (jj - 1));
        int hi = lo + jj;
        bool asc = (lo & k) == 0;
        int klo = keys[lo], khi = keys[hi];
        if ((klo > khi) == asc) {
          keys[lo] = khi;
          keys[hi] = klo;
        }
      }
      g.sync();
    }
  }
}

// ---- bitonic sort in registers -----------------------------------------------
// Sorts the 32·E values held by a full warp, E per lane in blocked layout
// (lane l holds elements l·E … l·E+E−1), ascending.  Partners closer than E
// are in the same lane (register exchange); farther ones are one shuffle away.
template <int E, typename U>
__device__ __forceinline__ void warp_bitonic_sort(U (&r)[E]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= E) {
        // partner in lane ^ (j/E); k > j >= E, so both direction bits of
        // element lane·E + i are bits of the lane: one decision per stage
        const bool asc = ((lane * E) & k) == 0;
        const bool lower = (lane & (j / E)) == 0;
        const bool keep_min = asc == lower;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const U other = __shfl_xor_sync(0xffffffffu, r[i], j / E);
          const U mn = r[i] < other ? r[i] : other;
          const U mx = r[i] < other ? other : r[i];
          r[i] = keep_min ? mn : mx;
        }
      } else {
        // partner in the same lane; element index bits below E come from i
        const bool lane_asc = ((lane * E) & k) == 0;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          if ((i & j) == 0) {
            const bool asc = (k < E) ? ((i & k) == 0) : lane_asc;
            const U x = r[i], y = r[i + j];
            const U mn = x < y ? x : y;
            const U mx = x < y ? y : x;
            r[i] = asc ? mn : mx;
            r[i + j] = asc ? mx : mn;
          }
        }
      }
    }
  }
}

// ---- stable LSD radix sort of 32-bit words in shared memory --------------------
template <int NW>
__device__ __forceinline__ void nw_sync() {
  if (NW == 1) __syncwarp();
  else __syncthreads();
}

// Sorts w[0..m) by the bit field [lo_bit, lo_bit + nbits) with DBITS-bit digits
// (5 to 8),
// least significant first, ping-ponging with tmp[0..m); returns the array
// that holds the result (w or tmp).  Bits outside the field travel with the
// word.  NW warps take part (NW = 1: the calling warp; NW > 1: the whole CTA
// of NW warps).  Per pass warp w owns the contiguous slice [w·S, w·S + S)
// (S = ⌈m/NW⌉ rounded up to 32): it counts its digits into cnt[d·NW + w],
// one exclusive scan over cnt (digit-major, so warp 0's 5s precede warp 1's
// 5s) gives every (digit, warp) its first output position, and each warp then
// scatters its slice 32 words at a time, ranking lanes with equal digits by
// ballots so equal digits keep their input order.  Each pass is
// therefore stable, and for distinct fields the result is ascending in the
// field.  cnt holds 2^DBITS·NW ints; scratch 33 ints (used when NW > 1).
template <int NW, int DBITS>
__device__ uint32_t* radix_sort_words(uint32_t* w, uint32_t* tmp, int m, int lo_bit, int nbits,
                                      int* cnt, int* scratch) {
  static_assert(DBITS >= 5 && DBITS <= 8, "digit width");
  constexpr int R = 1 << DBITS, PER = R / 32;  // counters owned by each thread
  constexpr uint32_t DM = R - 1;
  const int lane = threadIdx.x & 31;
  const int wid = NW == 1 ? 0 : (int)(threadIdx.x >> 5);
  const int tid = NW == 1 ? lane : (int)threadIdx.x;
  const int S = ((m + NW - 1) / NW + 31) & ~31;
  const int s0 = min(m, wid * S), s1 = min(m, s0 + S);
  uint32_t* src = w;
  uint32_t* dst = tmp;
  for (int sh = lo_bit; sh < lo_bit + nbits; sh += DBITS) {
#pragma unroll
    for (int k = 0; k < PER; ++k) cnt[tid * PER + k] = 0;
    nw_sync<NW>();
    for (int i = s0 + lane; i < s1; i += 32) atomicAdd(&cnt[((src[i] >> sh) & DM) * NW + wid], 1);
    nw_sync<NW>();
    int v[PER], sum = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      v[k] = cnt[tid * PER + k];
      sum += v[k];
    }
    int ex;
    if (NW == 1) {
      int incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      ex = incl - sum;
    } else {
      int tot;
      ex = block_exclusive_scan(sum, scratch, &tot);
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      cnt[tid * PER + k] = ex;
      ex += v[k];
    }
    nw_sync<NW>();
    for (int c = s0; c < s1; c += 32) {
      const int i = c + lane;
      const bool on = i < s1;
      const uint32_t x = on ? src[i] : 0u;
      const int d = on ? (int)((x >> sh) & DM) : R;
      // lanes with the same digit: one ballot per digit bit (and one for the
      // lanes in range), intersected (4% faster than __match_any_sync on the
      // 512-matrix batch)
      const unsigned on_mask = __ballot_sync(0xffffffffu, on);
      unsigned peers = on ? on_mask : ~on_mask;
#pragma unroll
      for (int b = 0; b < DBITS; ++b) {
        const bool bit = (d >> b) & 1;
        const unsigned bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
      }
      const int rank = __popc(peers & lanemask_lt());
      const int slot = on ? d * NW + wid : 0;
      const int base = on ? cnt[slot] : 0;
      __syncwarp();
      if (on && rank == 0) cnt[slot] = base + __popc(peers);
      __syncwarp();
      if (on) dst[base + rank] = x;
    }
    nw_sync<NW>();
    uint32_t* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

__host__ __device__ __forceinline__ int next_pow2_int(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

__host__ __device__ __forceinline__ int ilog2_int(int x) {  // x a power of two
  int l = 0;
  while ((1 << l) < x) ++l;
  return l;
}

}  // namespace spg
