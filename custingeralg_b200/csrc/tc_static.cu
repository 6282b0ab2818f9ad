// Static triangle count: degree orientation + vertex-grouped intersections (sm_100a).
//
// Replaces the reference's devicecuStingerAllTriangles (src/static_triangle_counting/cct.cu:216-270)
// and count_all_trianglesGPU (tests/cct_csr.cu:228-276). The reference intersects the full
// lists of every directed edge with a merge path split across 1-32 lanes and one block
// reduction per source vertex. Here:
//
//  1. Orientation (one pass). k_find_hubs registers the vertices with more than kHubMin = 256
//     neighbours (hubs); k_orient then builds the degree orientation G+ (u -> v iff
//     (deg u, u) < (deg v, v)) in the input's own index space: N+(u) is written, ascending by
//     id, at indp[start(u) ...], so no offsets scan is needed. Every triangle {x < y < z in
//     that order} is found exactly once: at x, on edge x->y, as the common element z of N+(x)
//     and N+(y). Warps take hub chunks of up to 2048 entries from one queue (the warp that
//     finishes a hub's last chunk moves the pieces together), then tiles of 32 vertex ids from
//     another, walking a tile's concatenated lists (at most 32 x 256 entries), so neither a
//     degree-64k hub nor a run of low-id vertices of degree 2000 (R-MAT) is one warp's serial
//     tail. The same pass
//     checks the input (ids in range, strictly ascending lists, no self-loops, a signed edge
//     checksum for symmetry) and fills the work queues of the count.
//  2. Counting. Every edge {c, o} is intersected once, at its centre c: the endpoint with the
//     larger out-degree (ties to the smaller id). The centre's N+(c) is a shared-memory hash set
//     of 4-slot buckets; the other list N+(o), the shorter one, goes through it, so the probe
//     work is the sum over edges of min(d+u, d+v). k_count is a persistent grid; a centre walks
//     its original neighbour list N(c) in groups of 32 and takes the neighbours it is centre
//     for. Tiers by a = d+(c):
//       CTA   a > warp_max: one CTA per item of 4096 neighbours, N+(c) staged in the full
//             2048-slot table (load <= 0.25 up to 512 entries) in passes of at most 1024
//             entries split evenly; a pass holds a value range of N+(c), and each streamed list
//             is cut to that range by binary search, so no list entry is probed twice;
//       warp  1 <= a <= warp_max (at most 128): one warp per centre (items of 256 neighbours for
//             centres with more), a warp-private set of up to 256 slots.
//     CTAs of 4 warps, 12 resident per SM (40 registers, 16 KB of shared memory each).
//     Per edge, the warp streams N+(o) with coalesced loads (four per lane in flight); or, for
//     short lists, one lane walks it while the other lanes walk theirs; or, for mid-size lists,
//     the warp walks all such lists of its group of neighbours concatenated (packed); the
//     scheduler (thresholds or learned per-degree-cell table) picks.
//  3. Attribution. Per-vertex counts never take a global atomic per triangle: the centre's count
//     stays in registers, the other endpoint's is reduced once per list (one redux.sync), and
//     the third vertex's is a shared-memory counter beside the hash slot that the probe found;
//     they flush with at most one global atomic per edge or staged entry. The triangle total
//     takes one global atomic per CTA.
#include <algorithm>
#include <climits>
#include <cstring>

#include "tc_internal.cuh"

#ifdef TC_DEBUG_PROGRESS
extern "C" void* tc_dbg_progress_host_dev;
extern "C" size_t tc_dbg_progress_bytes;
#endif

namespace tc {

namespace {

constexpr int kThreads = 128;     // 4 warps: small CTAs keep more warps resident per SM
constexpr int kWarps = kThreads / kWarp;
constexpr int kChunk = 1024;      // A entries staged per pass for an L-tier vertex
constexpr int kHashMax = 2048;    // hash slots for such a chunk (load <= 0.5)
constexpr int kUnroll = 4;        // list elements a lane loads before probing (independent loads)
constexpr int kWarpRange = 256;   // neighbours of a warp-tier centre per work item
constexpr int kCtaRange = 4096;   // neighbours of a CTA-tier centre per work item
static_assert(kWarpRange >= kItemRangeMin && kCtaRange >= kItemRangeMin, "queue sizing");
constexpr int kMedSlots = 2 * kWarpTierMax;  // warp-private hash slots (load <= 0.25 up to a = 64, else <= 0.5)
// Hash sets are bucketized: 4 slots per 16-byte bucket, probed with one 128-bit shared load,
// so a lookup ends after one bucket unless that bucket is full (rare at these loads).
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

#ifdef TC_DEBUG_PROGRESS
// Debug builds only: per-warp progress words and per-kernel entry/exit counters in host-mapped
// memory, readable while a kernel runs.
__device__ unsigned long long* tc_dbg_progress = nullptr;
__device__ unsigned long long* tc_dbg_kern = nullptr;
#define TC_DBG_MARK(idx, val)                                                              \
  do {                                                                                     \
    if (tc_dbg_progress) ((volatile unsigned long long*)tc_dbg_progress)[(idx)] = (val);  \
  } while (0)
#define TC_DBG_ENTER(id)                                                                     \
  do {                                                                                       \
    if (tc_dbg_kern && threadIdx.x == 0) atomicAdd_system(&tc_dbg_kern[2 * (id)], 1ull);      \
  } while (0)
#define TC_DBG_EXIT(id)                                                                      \
  do {                                                                                       \
    if (tc_dbg_kern && threadIdx.x == 0) atomicAdd_system(&tc_dbg_kern[2 * (id) + 1], 1ull);  \
  } while (0)
#else
#define TC_DBG_MARK(idx, val) \
  do {                        \
  } while (0)
#define TC_DBG_ENTER(id) \
  do {                   \
  } while (0)
#define TC_DBG_EXIT(id) \
  do {                  \
  } while (0)
#endif

// Hash sets of staged entries of N+(c). The third-vertex counter of an entry sits beside its
// slot: cnt[s] counts the triangles found through the key hkeys[s], so a hit adds to the slot
// it found with no indirection. Warp-private set (warp tier):
struct WarpTable {
  alignas(16) int32_t hkeys[kMedSlots];
  uint32_t cnt[kMedSlots];
};

// CTA-shared set of one chunk of a CTA-tier centre's N+(c) (16 KB):
struct BlockTable {
  alignas(16) int32_t hkeys[kHashMax];
  uint32_t cnt[kHashMax];
};

// Dynamic shared memory of k_count, laid out as CountSmem.
extern __shared__ __align__(16) unsigned char smem_raw[];

struct CountSmem {
  union {
    BlockTable L;
    WarpTable W[kWarps];
  } t;
  unsigned long long tri[kWarps];
  unsigned long long item;
  uint64_t mbar;  // completion of the bulk copy that stages a CTA-tier chunk
  int gctr;
  // Value range [vlo, vhi) of the CTA-tier pass in flight when its centre takes several passes
  // (ranged = 1; 0 for a centre of one pass). Only the CTA tier reads them.
  int ranged;
  int32_t vlo, vhi;
};

// ---- bulk copies into shared memory (cp.async.bulk, completion on an mbarrier) ----------------

// Bound of the wait for a staged chunk: it lands within microseconds; a wait that runs out sets
// kBadTimeout and the CTA stops (after a second bounded wait for its copy in flight).
constexpr unsigned long long kStageWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Issue one 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to shared memory; the mbarrier's phase completes when the bytes have landed.
__device__ __forceinline__ void stage_bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Wait (bounded by kStageWaitNs of device time) for the mbarrier phase `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (unsigned it = 0; it < (1u << 26); ++it) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > kStageWaitNs) break;
  }
  return false;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint64_t sym_hash(uint32_t x, uint32_t y) {
  uint64_t z = ((uint64_t)x << 32) | y;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

__device__ __forceinline__ uint32_t hash_bucket(int32_t key, int bbits) {
  return ((uint32_t)key * 0x9E3779B1u) >> (32 - bbits);
}

// Insert key (unique) into a table of 2^bbits buckets of 4 slots (load <= 0.5, so a bucket with
// a free slot is always found within 2^bbits steps). Slots of a bucket fill in order and are
// never freed, so a key that moved on found every slot before it taken.
__device__ __forceinline__ void hash_insert(int32_t* keys, int bbits, int32_t key) {
  const uint32_t bmask = (1u << bbits) - 1;
  uint32_t b = hash_bucket(key, bbits);
  for (uint32_t it = 0; it <= bmask; ++it) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int32_t prev = atomicCAS(&keys[4 * b + t], -1, key);
      if (prev == -1 || prev == key) return;
    }
    b = (b + 1) & bmask;
  }
}

// Continue a lookup whose first bucket b was full and lacked key: slot of key, or -1.
__device__ __forceinline__ int hash_find_after(const int32_t* keys, int bbits, int32_t key, uint32_t b) {
  const uint32_t bmask = (1u << bbits) - 1;
  for (uint32_t it = 0; it < bmask; ++it) {
    b = (b + 1) & bmask;
    const int4 q = *reinterpret_cast<const int4*>(keys + 4 * b);
    if (q.x == key) return 4 * b;
    if (q.y == key) return 4 * b + 1;
    if (q.z == key) return 4 * b + 2;
    if (q.w == key) return 4 * b + 3;
    if (q.w == -1) return -1;
  }
  return -1;
}

__device__ __forceinline__ int log2_cell(int x) {
  const int c = 31 - __clz(max(x, 1));
  return min(c, 15);
}

// Weights a found triangle (u, v, w) adds to each vertex's per-vertex output.
// TC_PV_HANDLE: 1 each (doubled at flush: out = 2 t(v)).
// TC_PV_CSR: the reference's raw-CSR kernel counts a triangle at every edge (x, y) with
// y > x whose lists share the third vertex, crediting x: the smallest id gets 2, the middle 1.
template <int PV>
__device__ __forceinline__ void tri_weights(int32_t u, int32_t v, int32_t w, uint32_t& wu, uint32_t& wv,
                                            uint32_t& ww) {
  if (PV == TC_PV_CSR) {
    wu = (u < v) + (u < w);
    wv = (v < u) + (v < w);
    ww = (w < u) + (w < v);
  } else {
    wu = wv = ww = 1u;
  }
}

template <int PV>
__host__ __device__ constexpr uint32_t flush_mult() {
  return PV == TC_PV_HANDLE || PV == TC_PV_HANDLE64 ? 2u : 1u;
}

// Handle conventions (every triangle weighs 1 per vertex, doubled at flush): int32 or int64 output.
template <int PV>
__host__ __device__ constexpr bool handle_like() {
  return PV == TC_PV_HANDLE || PV == TC_PV_HANDLE64;
}

// Flush x triangles (weights) of vertex v into the per-vertex output: int32 entries, or int64
// entries for TC_PV_HANDLE64 (the output pointer then addresses int64[nv]).
template <int PV>
__device__ __forceinline__ void out_add(uint32_t* __restrict__ out, const int32_t v, const uint32_t x) {
  if (PV == TC_PV_HANDLE64)
    atomicAdd(reinterpret_cast<unsigned long long*>(out) + v, (unsigned long long)x * flush_mult<PV>());
  else
    atomicAdd(out + v, x * flush_mult<PV>());
}

// Is the edge {c, o} intersected at c? At the endpoint with the larger out-degree (its list is
// the hash set, the other one is streamed), ties to the smaller id. Both endpoints read the same
// dplus values, so exactly one of them takes the edge.
__device__ __forceinline__ bool centre_of(int32_t c, int a, int32_t o, int b) {
  return b < a || (b == a && c < o);
}

// Probe one entry key of the list owned by o into the hash set; returns 1 on a hit. Per hit, the
// third vertex's counter cnt[slot] gets its weight; vacc and c_acc collect the weights of
// o and of the centre c (TC_PV_CSR only: in handle mode all weights are 1 and the caller counts
// the hits instead).
template <int PV>
__device__ __forceinline__ uint32_t probe_one(const int32_t key, const int32_t c, const int32_t o,
                                              const int32_t* hkeys, const int bits, uint32_t* cnt,
                                              uint32_t& c_acc, uint32_t& vacc) {
  // First bucket in one 128-bit load; the common case (a miss in a bucket with a free slot)
  // ends here without computing a slot.
  const uint32_t bk = hash_bucket(key, bits);
  const int4 q = *reinterpret_cast<const int4*>(hkeys + 4 * bk);
  const bool hit = (q.x == key) | (q.y == key) | (q.z == key) | (q.w == key);
  if (!(hit | (q.w != -1))) return 0;
  const int s = hit ? (int)(4 * bk) + (q.x == key ? 0 : q.y == key ? 1 : q.z == key ? 2 : 3)
                    : hash_find_after(hkeys, bits, key, bk);
  if (s < 0) return 0;
  if (handle_like<PV>()) {
    atomicAdd(&cnt[s], 1u);
  } else if (PV == TC_PV_CSR) {
    uint32_t wc, wo, ww;
    tri_weights<PV>(c, o, key, wc, wo, ww);
    c_acc += wc;
    vacc += wo;
    if (ww) atomicAdd(&cnt[s], ww);
  }
  return 1;
}

// The warp streams the list lst[0 .. len) through the hash set with coalesced loads, kUnroll
// per lane in flight; returns this lane's hits.
template <int PV>
__device__ __forceinline__ uint32_t probe_list(const int32_t* __restrict__ lst, const int len, const int32_t c,
                                               const int32_t o, const int32_t* hkeys, const int bits,
                                               uint32_t* cnt, uint32_t& c_acc, uint32_t& vacc) {
  const int lane = threadIdx.x & (kWarp - 1);
  uint32_t hits = 0;
  for (int k0 = lane; k0 < len; k0 += kUnroll * kWarp) {
    int32_t w[kUnroll];
#pragma unroll
    for (int j = 0; j < kUnroll; ++j) {
      const int k = k0 + j * kWarp;
      w[j] = k < len ? __ldg(lst + k) : -1;
    }
#pragma unroll
    for (int j = 0; j < kUnroll; ++j) {
      const int32_t key = w[j];
      if (key < 0) continue;
      // First bucket in one 128-bit load; the common case (a miss in a bucket with a free
      // slot) ends here without computing a slot.
      const uint32_t bk = hash_bucket(key, bits);
      const int4 q = *reinterpret_cast<const int4*>(hkeys + 4 * bk);
      const bool hit = (q.x == key) | (q.y == key) | (q.z == key) | (q.w == key);
      if (hit | (q.w != -1)) {
        const int s = hit ? (int)(4 * bk) + (q.x == key ? 0 : q.y == key ? 1 : q.z == key ? 2 : 3)
                          : hash_find_after(hkeys, bits, key, bk);
        if (s >= 0) {
          ++hits;
          if (handle_like<PV>()) {
            atomicAdd(&cnt[s], 1u);
          } else if (PV == TC_PV_CSR) {
            uint32_t wc, wo, ww;
            tri_weights<PV>(c, o, key, wc, wo, ww);
            c_acc += wc;
            vacc += wo;
            if (ww) atomicAdd(&cnt[s], ww);
          }
        }
      }
    }
  }
  return hits;
}

// One lane walks a whole (short) list lst[0 .. len), kUnroll entries in flight; returns the
// hits. The lanes of a warp walk different lists at once, so short lists do not leave most of
// the warp idle.
template <int PV>
__device__ __forceinline__ uint32_t walk_list(const int32_t* __restrict__ lst, const int len, const int32_t c,
                                              const int32_t o, const int32_t* hkeys, const int bits,
                                              uint32_t* cnt, uint32_t& c_acc, uint32_t& vacc) {
  uint32_t hits = 0;
  for (int k0 = 0; k0 < len; k0 += kUnroll) {
    int32_t w[kUnroll];
#pragma unroll
    for (int j = 0; j < kUnroll; ++j) w[j] = k0 + j < len ? __ldg(lst + k0 + j) : -1;
#pragma unroll
    for (int j = 0; j < kUnroll; ++j)
      if (w[j] >= 0) hits += probe_one<PV>(w[j], c, o, hkeys, bits, cnt, c_acc, vacc);
  }
  return hits;
}

// First index of the ascending list lst[0 .. len) whose entry is >= key (one lane, binary search).
__device__ __forceinline__ int lower_bound_list(const int32_t* __restrict__ lst, int len, const int32_t key) {
  int lo = 0;
  while (len > 0) {
    const int half = len >> 1;
    if (__ldg(lst + lo + half) < key) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}

// Lists at most this long are walked whole in a value-range pass (entries outside the pass's
// range just miss the hash set); longer ones are first cut to the range by two binary searches.
constexpr int kRangeSearchMin = 32;

// One warp takes the neighbours o = nbr[0 .. gcount) of centre c (out-degree a) and
// intersects every edge {c, o} whose centre is c: N+(o), the shorter list (b <= a entries), goes
// through the hash set of the staged chunk of N+(c) (2^bits buckets, cnt[slot] the counter of
// the key in that slot). Per edge the scheduler picks how (table cell, else the thresholds
// b <= lane_max, b <= packed_max):
//   lane:   each such lane walks its own list, all at once (short lists);
//   packed: the warp walks all such lists of the group concatenated, 32 entries per step (the
//           owner of an entry by binary search over the lanes' length prefix), so a group of
//           mid-size lists takes a few rounds of coalesced loads instead of one per list;
//   warp:   the lists are taken one at a time and the warp streams each with coalesced loads,
//           so o, its list and its count stay warp-uniform.
// When the hash set holds only the entries of N+(c) in [vlo, vhi) (one pass of a centre whose
// N+(c) is larger than a table), only the part of each N+(o) inside that range is walked: both
// lists are ascending, so no entry outside it can hit. The range sits in shared memory
// (CountSmem::ranged, vlo, vhi), so it holds no register across the group loop; kMayRange (the
// CTA tier) compiles the cut in, the warp tiers (one pass always) leave it out.
template <int PV, bool kMayRange>
__device__ __forceinline__ void process_group(const int32_t n, const int32_t c, const int a,
                                              const int32_t* __restrict__ nbr, const int gcount,
                                              const int32_t* hkeys, const int bits, uint32_t* cnt, const int32_t* __restrict__ dplus,
                                              const int64_t* __restrict__ offp, const int32_t* __restrict__ indp,
                                              uint32_t* __restrict__ out, const SchedParams& sp, uint32_t& tri,
                                              uint32_t& c_acc) {
  const int lane = threadIdx.x & (kWarp - 1);
  int32_t o = lane < gcount ? __ldg(nbr + lane) : -1;
  const bool valid = o >= 0 && o < n;  // ids out of range were flagged by the orientation
  if (!valid) o = 0;
  const int b = valid ? __ldg(dplus + o) : 0;
  const bool mine = valid && b > 0 && centre_of(c, a, o, b) &&
                    (sp.cell_filter == -1 ||
                     (sp.cell_filter >= 0 && log2_cell(a) * 16 + log2_cell(b) == sp.cell_filter));
  int64_t base = mine ? __ldg(offp + o) : 0;
  int strat = !mine ? -1
              : sp.use_table ? sp.table[log2_cell(a)][log2_cell(b)]
                             : (b <= sp.lane_max ? 1 : b <= sp.packed_max ? 2 : 0);
  int len = b;  // entries of N+(o) walked, from indp[base]
  const CountSmem& sm = *reinterpret_cast<const CountSmem*>(smem_raw);
  if (kMayRange && sm.ranged) {  // uniform over the CTA
    if (strat >= 0 && b > kRangeSearchMin) {
      const int32_t vlo = sm.vlo, vhi = sm.vhi;
      const int32_t* lst = indp + base;
      const int p0 = vlo == INT_MIN ? 0 : lower_bound_list(lst, b, vlo);
      const int p1 = vhi == INT_MAX ? b : p0 + lower_bound_list(lst + p0, b - p0, vhi);
      base += p0;
      len = p1 - p0;
      if (len == 0) strat = -1;
    }
    __syncwarp();
  }
  const bool by_lane = strat == 1;
  const bool by_pack = strat == 2;
  if (__any_sync(kFull, by_lane)) {
    if (by_lane) {
      uint32_t vacc = 0;
      const uint32_t hits = walk_list<PV>(indp + base, len, c, o, hkeys, bits, cnt, c_acc, vacc);
      tri += hits;
      if (handle_like<PV>()) {
        c_acc += hits;
        vacc = hits;
      }
      if (PV != TC_PV_NONE && vacc) out_add<PV>(out, o, vacc);
    }
    __syncwarp();
  }
  if (__any_sync(kFull, by_pack)) {
    const int len_l = by_pack ? len : 0;
    int incl = len_l;
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += y;
    }
    const int excl_l = incl - len_l;
    const int total = __shfl_sync(kFull, incl, kWarp - 1);
    for (int k0 = 0; k0 < total; k0 += kWarp) {
      const int k = k0 + lane;
      const bool in = k < total;
      int i = 0;  // owner lane: the largest i with excl_i <= k (its list is non-empty)
#pragma unroll
      for (int step = kWarp / 2; step > 0; step >>= 1) {
        const int e = __shfl_sync(kFull, excl_l, i + step);  // i + step <= 31
        if (e <= k) i += step;
      }
      const int64_t pbase = __shfl_sync(kFull, base, i);
      const int pos = k - __shfl_sync(kFull, excl_l, i);
      const int32_t po = __shfl_sync(kFull, o, i);
      const int32_t key = in ? __ldg(indp + pbase + pos) : -1;
      uint32_t vw = 0;  // o's weight of this entry's triangle
      const uint32_t h = key >= 0 ? probe_one<PV>(key, c, po, hkeys, bits, cnt, c_acc, vw) : 0u;
      tri += h;
      if (handle_like<PV>()) {
        c_acc += h;
        vw = h;
      }
      if (PV != TC_PV_NONE) {
        // o's counter: the first lane of each list's segment in this step adds the segment's sum
        const bool head = in && (pos == 0 || lane == 0);
        const unsigned heads = __ballot_sync(kFull, head);
        const unsigned w0 = __ballot_sync(kFull, vw & 1u);
        const unsigned w1 = PV == TC_PV_CSR ? __ballot_sync(kFull, vw & 2u) : 0u;
        if (head && (w0 | w1)) {
          const unsigned above = heads & ~((2u << lane) - 1u);  // heads of later lanes (lane 31: none)
          const unsigned seg = (above ? (1u << (__ffs(above) - 1)) - 1u : ~0u) & ~((1u << lane) - 1u);
          const uint32_t sum = __popc(w0 & seg) + 2u * __popc(w1 & seg);
          if (sum) out_add<PV>(out, po, sum);
        }
      }
    }
    __syncwarp();
  }
  unsigned todo = __ballot_sync(kFull, strat == 0);
  while (todo) {
    const int sl = __ffs(todo) - 1;
    todo &= todo - 1;
    const int32_t so = __shfl_sync(kFull, o, sl);
    const int sb = __shfl_sync(kFull, len, sl);
    const int64_t sbase = __shfl_sync(kFull, base, sl);
    uint32_t vacc = 0;
    const uint32_t hits = probe_list<PV>(indp + sbase, sb, c, so, hkeys, bits, cnt, c_acc, vacc);
    tri += hits;
    if (handle_like<PV>()) {
      c_acc += hits;
      vacc = hits;
    }
    if (PV != TC_PV_NONE) {
      vacc = __reduce_add_sync(kFull, vacc);
      if (lane == 0 && vacc) out_add<PV>(out, so, vacc);
    }
  }
  __syncwarp();
}

// One warp counts the edges of centre c (out-degree a <= kWarpTierMax) among its neighbours
// N(c)[k0 .. k1).
template <int PV>
__device__ __forceinline__ void warp_centre(const int32_t n, const int32_t c, const int a, const int64_t start,
                                            const int k0, const int k1, WarpTable& t,
                                            const int32_t* __restrict__ ind, const int32_t* __restrict__ dplus,
                                            const int64_t* __restrict__ offp, const int32_t* __restrict__ indp,
                                            uint32_t* __restrict__ out, const SchedParams& sp, uint32_t& tri) {
  const int lane = threadIdx.x & (kWarp - 1);
  int bits = 4;  // buckets: 4 * 2^bits slots >= 4a (load <= 0.25) while they fit in kMedSlots
  while ((1 << bits) < a && (8 << bits) <= kMedSlots) ++bits;
  const int S = 4 << bits;
  for (int s = lane; s < S; s += kWarp) {
    t.hkeys[s] = -1;
    t.cnt[s] = 0;
  }
  __syncwarp();
  for (int j = lane; j < a; j += kWarp) hash_insert(t.hkeys, bits, __ldg(indp + start + j));
  __syncwarp();
  uint32_t c_acc = 0;
  for (int g = k0; g < k1; g += kWarp)
    process_group<PV, false>(n, c, a, ind + start + g, min(kWarp, k1 - g), t.hkeys, bits, t.cnt, dplus, offp, indp,
                             out, sp, tri, c_acc);
  if (PV != TC_PV_NONE) {
    for (int s = lane; s < S; s += kWarp) {
      const uint32_t x = t.cnt[s];
      if (x) out_add<PV>(out, t.hkeys[s], x);
    }
    __syncwarp();
    c_acc = __reduce_add_sync(kFull, c_acc);
    if (lane == 0 && c_acc) out_add<PV>(out, c, c_acc);
  }
  __syncwarp();
}

// Work items of the queues: centre c and the first neighbour index k0 of its range of N(c).
__device__ __forceinline__ unsigned long long make_item(int32_t c, int32_t k0) {
  return ((unsigned long long)(uint32_t)c << 32) | (uint32_t)k0;
}

template <int PV>
__global__ void __launch_bounds__(kThreads, 12) k_count(const int32_t n, const int32_t* __restrict__ ind,
                                                    const int32_t* __restrict__ degv,
                                                    const int32_t* __restrict__ dplus,
                                                    const int64_t* __restrict__ offp,
                                                    const int32_t* __restrict__ indp,
                                                    const unsigned long long* __restrict__ large,
                                                    const unsigned long long* __restrict__ medium,
                                                    uint32_t* __restrict__ out, DevStatus* __restrict__ st,
                                                    const SchedParams sp) {
  TC_DBG_ENTER(6);
  CountSmem& sm = *reinterpret_cast<CountSmem*>(smem_raw);
  const int lane = threadIdx.x & (kWarp - 1);
  const int wid = threadIdx.x / kWarp;
  uint32_t tri = 0;
  const unsigned n_large = st->n_large;
  const unsigned n_medium = st->n_medium;

  // CTA tier: one CTA per item (centre with a > warp_max, kCtaRange of its neighbours), over
  // chunks of kChunk entries of N+(c), each staged into shared memory by one bulk copy.
  BlockTable& L = sm.t.L;
  if (threadIdx.x == 0) {
    mbar_init(&sm.mbar);
    sm.ranged = 0;
  }
  __syncthreads();
  uint32_t stage_phase = 0;
  while (true) {
    if (threadIdx.x == 0) {
      const unsigned q = atomicAdd(&st->q_large, 1u);
      sm.item = q < n_large ? large[q] : ~0ull;
    }
    __syncwarp();
    __syncthreads();
    const unsigned long long item = sm.item;
    __syncthreads();
    if (item == ~0ull) break;
    const int32_t c = (int32_t)(item >> 32);
    const int32_t k0 = (int32_t)(uint32_t)item;
    const int32_t a = dplus[c];
    const int64_t start = offp[c];
    const int32_t k1 = min(degv[c], k0 + kCtaRange);
    uint32_t c_acc = 0;
    // N+(c) in passes of at most kChunk entries, split evenly; pass pk holds the entries of N+(c)
    // in [vlo, vhi), and only that part of each streamed list is walked in it.
    const int passes = (a + kChunk - 1) / kChunk;
    for (int pk = 0; pk < passes; ++pk) {
      const int cb = (int)(((int64_t)pk * a) / passes);
      const int cb_next = (int)(((int64_t)(pk + 1) * a) / passes);
      const int clen = cb_next - cb;
      // the whole table whatever clen: load clen / kHashMax (<= 0.25 up to 512 entries, <= 0.5)
      constexpr int bits = 9;
      static_assert((4 << bits) == kHashMax, "CTA table size");
      const int S = 4 << bits;
      // Stage N+(c)[cb, cb + clen) in the counter half of the table (cleared after the build):
      // one bulk copy of the 16-byte units that cover it (at most clen + 3 entries, inside the
      // list or the array's padding), issued while the threads clear the keys.
      const int64_t gs = start + cb, ga = gs & ~int64_t(3);
      const int skip = (int)(gs - ga);
      static_assert(sizeof(L.cnt) >= sizeof(int32_t) * (kChunk + 4), "staging area");
      int32_t* stage = reinterpret_cast<int32_t*>(L.cnt);
      if (threadIdx.x == 0) {
        sm.gctr = 0;
        stage_bulk(stage, indp + ga, (uint32_t)(((skip + clen + 3) & ~3) * sizeof(int32_t)), &sm.mbar);
      }
      for (int s = threadIdx.x; s < S; s += kThreads) L.hkeys[s] = -1;
      const bool landed = mbar_wait(&sm.mbar, stage_phase);
      stage_phase ^= 1u;
      if (__syncthreads_or(!landed)) {
        // the copy did not land in time: report it, wait once more for it, stop this CTA
        if (threadIdx.x == 0) atomicOr(&st->bad_flags, kBadTimeout);
        mbar_wait(&sm.mbar, stage_phase ^ 1u);
        return;
      }
      if (threadIdx.x == 0) {
        sm.ranged = passes > 1;
        sm.vlo = pk == 0 ? INT_MIN : stage[skip];
        sm.vhi = pk + 1 == passes ? INT_MAX : __ldg(indp + start + cb_next);
      }
      for (int j = threadIdx.x; j < clen; j += kThreads) hash_insert(L.hkeys, bits, stage[skip + j]);
      __syncwarp();
      __syncthreads();
      for (int s = threadIdx.x; s < S; s += kThreads) L.cnt[s] = 0;
      __syncwarp();
      __syncthreads();
      const int ngroups = (k1 - k0 + kWarp - 1) / kWarp;
      while (true) {
        int g = 0;
        if (lane == 0) g = atomicAdd(&sm.gctr, 1);
        __syncwarp();
        g = __shfl_sync(kFull, g, 0);
        if (g >= ngroups) break;
        const int gk = k0 + g * kWarp;
        process_group<PV, true>(n, c, a, ind + start + gk, min(kWarp, k1 - gk), L.hkeys, bits, L.cnt, dplus, offp,
                                indp, out, sp, tri, c_acc);
      }
      __syncwarp();
      __syncthreads();
      if (PV != TC_PV_NONE) {
        for (int s = threadIdx.x; s < S; s += kThreads) {
          const uint32_t x = L.cnt[s];
          if (x) out_add<PV>(out, L.hkeys[s], x);
        }
      }
      __syncwarp();
      __syncthreads();
    }
    if (threadIdx.x == 0) sm.ranged = 0;  // the next item sets it again before its first group
    if (PV != TC_PV_NONE) {
      c_acc = __reduce_add_sync(kFull, c_acc);
      if (lane == 0 && c_acc) out_add<PV>(out, c, c_acc);
    }
  }

  // From here every warp works alone, on its own slice of the (now free) staging area.
  WarpTable& W = sm.t.W[wid];

  // Warp tier, centres with many neighbours: one warp per item (kWarpRange neighbours).
  while (true) {
    unsigned long long item = ~0ull;
    if (lane == 0) {
      const unsigned q = atomicAdd(&st->q_medium, 1u);
      if (q < n_medium) item = medium[q];
    }
    __syncwarp();
    item = __shfl_sync(kFull, item, 0);
    if (item == ~0ull) break;
    const int32_t c = (int32_t)(item >> 32);
    const int32_t k0 = (int32_t)(uint32_t)item;
    const int a = __ldg(dplus + c);
    const int64_t start = __ldg(offp + c);
    const int k1 = min(__ldg(degv + c), k0 + kWarpRange);
    warp_centre<PV>(n, c, a, start, k0, k1, W, ind, dplus, offp, indp, out, sp, tri);
  }

  // Warp tier, the rest (1 <= a <= warp_max, degree <= kWarpRange): one warp per centre,
  // claimed in chunks of vertex ids.
  while (true) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(&st->q_small, (unsigned long long)sp.chunk);
    __syncwarp();
    c0 = __shfl_sync(kFull, c0, 0);
    if (c0 >= (unsigned long long)n) break;
    const int32_t cend = (int32_t)min((unsigned long long)n, c0 + (unsigned long long)sp.chunk);
    // this count's centres (all of them unless sharded), read per claimed chunk
    const bool sharded = st->sharded != 0;
    const int32_t s_lo = (int32_t)st->shard_lo, s_hi = (int32_t)st->shard_hi;
    for (int32_t ub = (int32_t)c0; ub < cend; ub += kWarp) {
      const int32_t uu = ub + lane;
      const bool in = uu < cend;
      const int aa = in ? __ldg(dplus + uu) : 0;
      const int dd = in ? __ldg(degv + uu) : 0;
      unsigned elig = __ballot_sync(
          kFull, aa >= 1 && aa <= sp.warp_max && dd <= kWarpRange && (!sharded || (uu >= s_lo && uu < s_hi)));
      while (elig) {
        const int sl = __ffs(elig) - 1;
        elig &= elig - 1;
        const int32_t c = ub + sl;
        const int a = __shfl_sync(kFull, aa, sl);
        const int d = __shfl_sync(kFull, dd, sl);
        warp_centre<PV>(n, c, a, __ldg(offp + c), 0, d, W, ind, dplus, offp, indp, out, sp, tri);
      }
    }
  }

  // One global atomic per CTA for the triangle total.
  __syncwarp();
  const unsigned long long t = warp_sum((unsigned long long)tri);
  if (lane == 0) sm.tri[wid] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < kWarps; ++w) s += sm.tri[w];
    if (s) atomicAdd(&st->triangles, s);
  }
  TC_DBG_EXIT(6);
}

// ---- orientation ------------------------------------------------------------------------

__device__ __forceinline__ bool precedes(int32_t du, int32_t u, int32_t dv, int32_t v) {
  return du < dv || (du == dv && u < v);
}

// One warp orients entries [k_begin, k_end) of u's list (s = its start, d = its degree): it
// checks each entry (id in range, strictly ascending, no self-loop, signed symmetry checksum)
// and, when kWrite, writes the out-neighbours (in list order) to indp[out_base ...]. Returns
// their number (warp-uniform).
template <class View, bool kWrite>
__device__ __forceinline__ int orient_range(const View& g, const int32_t n, const int32_t u, const int32_t d,
                                            const int64_t s, const int32_t k_begin, const int32_t k_end,
                                            int32_t* __restrict__ indp, const int64_t out_base,
                                            unsigned long long& chk, unsigned& bad) {
  const int lane = threadIdx.x & (kWarp - 1);
  const unsigned lt = lanemask_lt();
  int cnt = 0;
  int32_t last = k_begin > 0 ? g.ind[s + k_begin - 1] : INT32_MIN;
  for (int32_t k0 = k_begin; k0 < k_end; k0 += kWarp) {
    const int32_t k = k0 + lane;
    const bool in = k < k_end;
    const int32_t v = in ? g.ind[s + k] : INT32_MAX;
    int32_t prev = __shfl_up_sync(kFull, v, 1);
    if (lane == 0) prev = last;
    last = __shfl_sync(kFull, v, kWarp - 1);
    bool pred = false;
    if (in) {
      if (v < 0 || v >= n) {
        bad |= kBadRange;
      } else {
        if (k > 0 && prev >= v) bad |= kBadOrder;
        if (v == u) bad |= kBadSelfLoop;
        pred = precedes(d, u, g.len(v), v);
        const uint64_t h = (u < v) ? sym_hash((uint32_t)u, (uint32_t)v) : sym_hash((uint32_t)v, (uint32_t)u);
        chk += (u < v) ? h : (0ull - h);
      }
    }
    __syncwarp();
    const unsigned msk = __ballot_sync(kFull, pred);
    if (kWrite && pred) indp[out_base + cnt + __popc(msk & lt)] = v;
    cnt += __popc(msk);
  }
  return cnt;
}

// Orientation bookkeeping of a finished vertex u with degree d and out-degree a (warp-uniform
// call): its offset, degree and out-degree and the work figures.
struct OrientAcc {
  unsigned long long work = 0, ei = 0;
  unsigned mx = 0;
};

__device__ __forceinline__ void finish_vertex(const int32_t u, const int32_t d, const int64_t s, const int32_t a,
                                              int32_t* __restrict__ dplus, int64_t* __restrict__ offp,
                                              int32_t* __restrict__ degv, OrientAcc& acc) {
  const int lane = threadIdx.x & (kWarp - 1);
  if (lane == 0) {
    dplus[u] = a;
    offp[u] = s;
    degv[u] = d;
    if (d >= 2) acc.ei += (unsigned long long)a;
    // sum over u -> v of d+(u) + d+(v) = sum over v of d+(v) deg(v)
    acc.work += (unsigned long long)a * (unsigned long long)d;
    acc.mx = max(acc.mx, (unsigned)a);
  }
}

// Register the vertices whose list is longer than kHubMin: they are oriented in chunks of up to
// kHubChunk entries that separate warps take. One thread per vertex. A hub starts with
// out-degree 0, so a hub that is never completed (capacity error) leaves nothing for the count
// to read.
template <class View>
__global__ void __launch_bounds__(256) k_find_hubs(const View g, const int32_t n, int32_t* __restrict__ dplus,
                                                   int64_t* __restrict__ offp, int32_t* __restrict__ degv,
                                                   int32_t* __restrict__ hub_u,
                                                   int32_t* __restrict__ hub_base, int32_t* __restrict__ hub_done,
                                                   int32_t* __restrict__ chunk_hub, const int64_t hub_cap,
                                                   const int64_t chunk_cap, DevStatus* __restrict__ st) {
  for (int64_t uu = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; uu < n; uu += (int64_t)gridDim.x * blockDim.x) {
    const int32_t u = (int32_t)uu;
    const int32_t d = g.len(u);
    if (d <= kHubMin) continue;
    dplus[u] = 0;
    offp[u] = 0;
    degv[u] = 0;
    const int nch = (d + kHubChunk - 1) / kHubChunk;
    const unsigned h = atomicAdd(&st->n_hubs, 1u);
    const unsigned base = atomicAdd(&st->n_hub_chunks, (unsigned)nch);
    const bool ok = h < hub_cap && (int64_t)base + nch <= chunk_cap;
    if (ok) {
      hub_u[h] = u;
      hub_base[h] = (int32_t)base;
      hub_done[h] = 0;
    } else {
      atomicOr(&st->bad_flags, kBadCapacity);
    }
    for (int c = 0; c < nch && (int64_t)base + c < chunk_cap; ++c) chunk_hub[base + c] = ok ? (int32_t)h : -1;
  }
}

// Single-pass orientation into the input's own index space: N+(u) is written at
// indp[start(u) ...], so no offsets scan is needed (offp[u] = start(u)). A persistent grid of
// warps first takes hub chunks from one queue, then tiles of vertex ids from another. A hub
// chunk is written at its own position in the hub's list; the warp that finishes a hub's last
// chunk (a counter per hub) moves the pieces together and completes the vertex.
template <class View, bool kWrite>
__global__ void __launch_bounds__(256) k_orient(const View g, const int32_t n, int32_t* __restrict__ dplus,
                                                int64_t* __restrict__ offp, int32_t* __restrict__ degv,
                                                int32_t* __restrict__ indp, const int64_t e_cap,
                                                const int32_t* __restrict__ hub_u,
                                                const int32_t* __restrict__ hub_base, int32_t* __restrict__ hub_cnt,
                                                int32_t* __restrict__ hub_done, const int32_t* __restrict__ chunk_hub,
                                                const int64_t hub_cap, const int64_t chunk_cap, DevStatus* __restrict__ st) {
  const int lane = threadIdx.x & (kWarp - 1);
  const unsigned nchunks = (unsigned)min((long long)st->n_hub_chunks, (long long)chunk_cap);
  const unsigned nhubs = (unsigned)min((long long)st->n_hubs, (long long)hub_cap);
  unsigned long long chk = 0;
  unsigned bad = 0;
  OrientAcc acc;

  // Hub chunks.
  while (true) {
    unsigned q = 0;
    if (lane == 0) q = atomicAdd(&st->q_orient_hub, 1u);
    __syncwarp();
    q = __shfl_sync(kFull, q, 0);
    if (q >= nchunks) break;
    const int h = chunk_hub[q];
    if (h < 0 || h >= (int)nhubs) continue;
    const int hb = hub_base[h];
    const int32_t u = hub_u[h];
    const int64_t s = g.start(u);
    const int32_t d = g.len(u);
    const int nch = (d + kHubChunk - 1) / kHubChunk;
    const int c = (int)q - hb;
    if (c < 0 || c >= nch) continue;
    if (s < 0 || s + d > e_cap) {
      bad |= kBadCapacity;
      continue;
    }
    const int32_t k_begin = c * kHubChunk, k_end = min(d, k_begin + kHubChunk);
    const int cnt = orient_range<View, kWrite>(g, n, u, d, s, k_begin, k_end, indp, s + k_begin, chk, bad);
    // Publish this chunk (entries written by every lane, then its count), then count it done.
    if (lane == 0) hub_cnt[q] = cnt;
    __threadfence();
    __syncwarp();
    int done = 0;
    if (lane == 0) done = atomicAdd(&hub_done[h], 1);
    __syncwarp();
    done = __shfl_sync(kFull, done, 0);
    if (done != nch - 1) continue;
    // Last chunk of this hub: gather the pieces (each chunk's out-neighbours start at the
    // chunk's own position; moving them down in chunk order never overwrites an unread entry).
    __threadfence();
    int a = 0;
    for (int cc = 0; cc < nch; ++cc) {
      const int cn = __ldcg(hub_cnt + hb + cc);
      if (kWrite && cc > 0 && cn > 0) {
        const int64_t src = s + (int64_t)cc * kHubChunk, dst = s + a;
        for (int k0 = 0; k0 < cn; k0 += kWarp) {
          const int k = k0 + lane;
          const int32_t x = k < cn ? __ldcg(indp + src + k) : 0;
          __syncwarp();
          if (k < cn) indp[dst + k] = x;
          __syncwarp();
        }
      }
      a += cn;
    }
    finish_vertex(u, d, s, a, dplus, offp, degv, acc);
  }

  // Vertex tiles (hubs skipped: done above). The warp walks the concatenated lists of a tile's
  // 32 vertices, 32 entries per step: short lists leave no lane idle, and a step is one round of
  // coalesced loads instead of one dependent round per vertex. Lane i keeps vertex t0 + i; the
  // owner of entry k is the last vertex whose list starts at or before k (a binary search over
  // the lanes' exclusive prefix of the lengths). An out-neighbour's rank in N+(u) is its vertex's
  // count from earlier steps (per-warp shared counter) plus the predecessors in its segment.
  constexpr int kTile = 32;
  __shared__ int32_t s_out[256 / kWarp][kTile];
  int32_t* const my_out = s_out[threadIdx.x / kWarp];
  const unsigned lt = lanemask_lt();
  while (true) {
    unsigned t0 = 0;
    if (lane == 0) t0 = atomicAdd(&st->q_orient_vtx, (unsigned)kTile);
    __syncwarp();
    t0 = __shfl_sync(kFull, t0, 0);
    if (t0 >= (unsigned)n) break;
    const int32_t u_l = (int32_t)t0 + lane;
    const bool in_t = u_l < n;
    const int32_t d_l = in_t ? g.len(u_l) : 0;
    const int64_t s_l = in_t ? g.start(u_l) : 0;
    const bool own_l = in_t && d_l <= kHubMin;  // hubs were completed by the chunk loop
    const bool cap_bad = own_l && (s_l < 0 || s_l + d_l > e_cap);
    if (cap_bad) bad |= kBadCapacity;
    const int32_t len_l = own_l && !cap_bad ? d_l : 0;
    int32_t incl = len_l;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
      const int32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const int32_t excl_l = incl - len_l;
    const int32_t total = __shfl_sync(kFull, incl, kWarp - 1);
    my_out[lane] = 0;
    __syncwarp();
    int32_t last = INT32_MIN;
    for (int32_t k0 = 0; k0 < total; k0 += kWarp) {
      const int32_t k = k0 + lane;
      const bool in = k < total;
      int i = 0;  // owner lane: the largest i with excl_i <= k (its list is non-empty)
#pragma unroll
      for (int step = kWarp / 2; step > 0; step >>= 1) {
        const int32_t e = __shfl_sync(kFull, excl_l, i + step);  // i + step <= 31
        if (e <= k) i += step;
      }
      const int32_t d = __shfl_sync(kFull, d_l, i);
      const int64_t s = __shfl_sync(kFull, s_l, i);
      const int32_t pos = k - __shfl_sync(kFull, excl_l, i);
      const int32_t u = (int32_t)t0 + i;
      const int32_t v = in ? g.ind[s + pos] : INT32_MAX;
      int32_t prev = __shfl_up_sync(kFull, v, 1);
      if (lane == 0) prev = last;
      last = __shfl_sync(kFull, v, kWarp - 1);
      bool pred = false;
      if (in) {
        if (v < 0 || v >= n) {
          bad |= kBadRange;
        } else {
          if (pos > 0 && prev >= v) bad |= kBadOrder;
          if (v == u) bad |= kBadSelfLoop;
          pred = precedes(d, u, g.len(v), v);
          const uint64_t h = (u < v) ? sym_hash((uint32_t)u, (uint32_t)v) : sym_hash((uint32_t)v, (uint32_t)u);
          chk += (u < v) ? h : (0ull - h);
        }
      }
      const unsigned msk = __ballot_sync(kFull, pred);
      const bool head = in && (pos == 0 || lane == 0);  // first entry of its vertex in this step
      const unsigned heads = __ballot_sync(kFull, head);
      const int seg0 = 31 - __clz(heads & (lt | (1u << lane)));
      const int prior = in ? my_out[i] : 0;
      __syncwarp();
      if (kWrite && pred) indp[s + prior + __popc(msk & lt & ~((1u << seg0) - 1u))] = v;
      if (head) {
        const unsigned above = heads & ~(lt | (1u << lane));
        const unsigned below_next = above ? ((1u << (__ffs(above) - 1)) - 1u) : ~0u;
        my_out[i] = prior + __popc(msk & below_next & ~((1u << lane) - 1u));
      }
      __syncwarp();
    }
    const int32_t a_l = own_l ? my_out[lane] : 0;
    __syncwarp();
    // Finish the tile's vertices, one per lane (the bookkeeping of finish_vertex).
    if (own_l) {
      dplus[u_l] = a_l;
      offp[u_l] = cap_bad ? 0 : s_l;
      degv[u_l] = cap_bad ? 0 : d_l;
      const int32_t dd = cap_bad ? 0 : d_l;
      if (dd >= 2) acc.ei += (unsigned long long)a_l;
      acc.work += (unsigned long long)a_l * (unsigned long long)dd;
      acc.mx = max(acc.mx, (unsigned)a_l);
    }
  }

  __syncwarp();
  chk = warp_sum(chk);
  acc.work = warp_sum(acc.work);
  acc.ei = warp_sum(acc.ei);
  acc.mx = __reduce_max_sync(kFull, acc.mx);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(kFull, bad, o);
  if (lane == 0) {
    if (chk) atomicAdd(&st->sym_checksum, chk);
    if (bad) atomicOr(&st->bad_flags, bad);
    if (acc.work) atomicAdd(&st->oriented_work, acc.work);
    if (acc.ei) atomicAdd(&st->edges_intersected, acc.ei);
    if (acc.mx) atomicMax(&st->max_dplus, acc.mx);
  }
}

// The count's work queues, filled after the orientation. A centre with out-degree a > warp_max
// gets CTA items of kCtaRange neighbours; one with a <= warp_max and more than kWarpRange
// neighbours gets warp items of kWarpRange (the other centres are claimed by id ranges). The CTA
// queue is ordered by estimated item work, largest first, so the persistent grid does not end
// on a few long items: the work class of a centre's items is log2(a * min(d, kCtaRange)), and
// classes are laid out in decreasing order, each in vertex-id order (which on R-MAT keeps
// centres with shared neighbours together). k_push_items counts the items per class and fills
// the warp queue; k_fill_items places the CTA items.
constexpr int kWorkClasses = 32;

__device__ __forceinline__ int work_class(const int32_t a, const int32_t d) {
  const unsigned long long w = (unsigned long long)a * (unsigned long long)min(d, kCtaRange);
  return min(kWorkClasses - 1, 63 - __clzll(max(w, 1ull)));
}

// Is u a centre of this count's shard (every centre when the count is not sharded)?
__device__ __forceinline__ bool in_shard(const DevStatus* __restrict__ st, const int32_t u) {
  return !st->sharded || (u >= (int32_t)st->shard_lo && u < (int32_t)st->shard_hi);
}

__device__ __forceinline__ bool cta_centre(const DevStatus* __restrict__ st, const int32_t u, const int32_t a,
                                           const int warp_max) {
  return a > warp_max && in_shard(st, u);
}

__global__ void __launch_bounds__(256) k_push_items(const int32_t n, const int32_t* __restrict__ dplus,
                                                    const int32_t* __restrict__ degv,
                                                    unsigned long long* __restrict__ medium, const int64_t item_cap,
                                                    DevStatus* __restrict__ st, const int warp_max) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) / kWarp;
  unsigned bad = 0;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; t * kWarp < n; t += nwarps) {
    const int64_t uu = t * kWarp + lane;
    const bool in = uu < n;
    const int32_t u = (int32_t)uu;
    const int32_t a = in ? dplus[u] : 0;
    const int32_t d = in ? degv[u] : 0;
    if (in && cta_centre(st, u, a, warp_max))
      atomicAdd(&st->cls_cnt[work_class(a, d)], (unsigned)((d + kCtaRange - 1) / kCtaRange));
    const bool wrp = in && a > 0 && a <= warp_max && d > kWarpRange && in_shard(st, u);
    const int x = wrp ? (d + kWarpRange - 1) / kWarpRange : 0;
    int incl = x;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
      const int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const int tot = __shfl_sync(kFull, incl, kWarp - 1);
    if (tot == 0) continue;
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&st->n_medium, (unsigned)tot);
    base = __shfl_sync(kFull, base, 0);
    if ((int64_t)base + tot > item_cap) {
      bad |= kBadCapacity;
      continue;
    }
    for (int j = 0; j < x; ++j) medium[base + (incl - x) + j] = make_item(u, j * kWarpRange);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(kFull, bad, o);
  if (lane == 0 && bad) atomicOr(&st->bad_flags, bad);
}

__global__ void __launch_bounds__(256) k_fill_items(const int32_t n, const int32_t* __restrict__ dplus,
                                                    const int32_t* __restrict__ degv,
                                                    unsigned long long* __restrict__ large, const int64_t item_cap,
                                                    DevStatus* __restrict__ st, const int warp_max) {
  __shared__ unsigned cls_base[kWorkClasses];
  __shared__ unsigned total;
  if (threadIdx.x < kWarp) {
    // exclusive scan over the classes in decreasing order: class c starts after all classes > c
    const int lane = threadIdx.x;
    const unsigned x = st->cls_cnt[kWorkClasses - 1 - lane];
    unsigned incl = x;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
      const unsigned y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    cls_base[kWorkClasses - 1 - lane] = incl - x;
    if (lane == kWarp - 1) total = incl;
  }
  __syncthreads();
  const unsigned n_items = (unsigned)min((long long)total, (long long)item_cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->n_large = n_items;
    if ((long long)total > item_cap) atomicOr(&st->bad_flags, kBadCapacity);
  }
  for (int64_t uu = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; uu < n; uu += (int64_t)gridDim.x * blockDim.x) {
    const int32_t u = (int32_t)uu;
    const int32_t a = dplus[u];
    if (!cta_centre(st, u, a, warp_max)) continue;
    const int32_t d = degv[u];
    const int cls = work_class(a, d);
    const int nit = (d + kCtaRange - 1) / kCtaRange;
    const unsigned at = cls_base[cls] + atomicAdd(&st->cls_pos[cls], (unsigned)nit);
    if ((int64_t)at + nit > (int64_t)n_items) continue;  // only past a capacity error
    for (int j = 0; j < nit; ++j) large[at + j] = make_item(u, j * kCtaRange);
  }
}

// ---- multi-GPU split of the static count -------------------------------------------------

// Predicted intersection work of each centre c (needs the orientation): one probe per entry of
// the other endpoint's list for every edge {c, o} that c is the centre of, plus 2 per such edge
// and 1 per neighbour scanned, in units of 16 (int32, clamped). One warp per vertex.
template <class View>
__global__ void __launch_bounds__(256) k_shard_cost(const View g, const int32_t n, const int32_t* __restrict__ dplus,
                                                    int32_t* __restrict__ cost) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) / kWarp;
  for (int64_t uu = gw; uu < n; uu += nw) {
    const int32_t u = (int32_t)uu;
    const int32_t d = g.len(u), a = dplus[u];
    const int64_t s = g.start(u);
    unsigned long long w = 0;
    for (int32_t k = lane; k < d; k += kWarp) {
      const int32_t o = g.ind[s + k];
      if (o < 0 || o >= n) continue;
      const int32_t b = dplus[o];
      if (b > 0 && centre_of(u, a, o, b)) w += (unsigned long long)b + 2ull;
    }
    w = warp_sum(w);
    if (lane == 0) cost[u] = (int32_t)min((w + (unsigned long long)d + 15ull) / 16ull, (unsigned long long)INT32_MAX);
  }
}

// This count's range of centres (shard_start over the exclusive prefix of the costs).
__global__ void k_shard_bounds(const int64_t* __restrict__ prefix, const int32_t n, const int32_t shard,
                               const int32_t nshards, DevStatus* __restrict__ st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int32_t lo = shard_start(prefix, n, shard, nshards), hi = shard_start(prefix, n, shard + 1, nshards);
  st->shard_lo = (unsigned)lo;
  st->shard_hi = (unsigned)hi;
  st->shard_work = (unsigned long long)(prefix[hi] - prefix[lo]);
  st->total_work = (unsigned long long)prefix[n];
  st->sharded = 1;
}

// ---- exclusive scan of int32 counts into int64 offsets ------------------------------------

__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(const int32_t* __restrict__ in, const int64_t n,
                                                                 int64_t* __restrict__ tile_sums) {
  TC_DBG_ENTER(2);
  __shared__ long long red[kScanThreads / kWarp];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  long long s = 0;
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / kWarp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < kScanThreads / kWarp; ++w) t += red[w];
    tile_sums[blockIdx.x] = t;
  }
  TC_DBG_EXIT(2);
}

// Single CTA: exclusive scan of tile_sums[0..ntiles) in place, total into tile_sums[ntiles].
__global__ void __launch_bounds__(1024) k_scan_tile_prefix(int64_t* __restrict__ tile_sums, const int64_t ntiles) {
  TC_DBG_ENTER(3);
  __shared__ long long wsum[32];
  __shared__ long long carry_s;
  const int lane = threadIdx.x & 31, wid = threadIdx.x / 32;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < ntiles; b0 += 1024) {
    const int64_t i = b0 + threadIdx.x;
    const long long x = (i < ntiles) ? tile_sums[i] : 0;
    long long incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      long long w = wsum[lane];
      long long wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(kFull, wi, o);
        if (lane >= o) wi += t;
      }
      wsum[lane] = wi - w;
    }
    __syncthreads();
    const long long c = carry_s;
    if (i < ntiles) tile_sums[i] = c + wsum[wid] + incl - x;
    __syncthreads();
    if (threadIdx.x == 1023) carry_s = c + wsum[wid] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sums[ntiles] = carry_s;
  TC_DBG_EXIT(3);
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int32_t* __restrict__ in, const int64_t n,
                                                             const int64_t* __restrict__ tile_sums,
                                                             int64_t* __restrict__ out, const int64_t ntiles) {
  TC_DBG_ENTER(4);
  __shared__ long long wsum[kScanThreads / kWarp];
  const int lane = threadIdx.x & 31, wid = threadIdx.x / 32;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
  long long v[kScanPer];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t i = base + k;
    v[k] = (i < n) ? in[i] : 0;
    s += v[k];
  }
  long long incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  long long wpre = 0;
  for (int w = 0; w < wid; ++w) wpre += wsum[w];
  long long run = tile_sums[blockIdx.x] + wpre + incl - s;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int64_t i = base + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[ntiles];
  TC_DBG_EXIT(4);
}

int orient_grid(int64_t n) {
  const int64_t want = (n + kWarps - 1) / kWarps;
  const int64_t cap = (int64_t)device_info().sms * 16;
  return (int)std::max<int64_t>(1, std::min(want, cap));
}

int hubs_grid(int64_t n) {
  const int64_t want = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)device_info().sms * 8));
}

template <int PV>
tc_status launch_count(int32_t n, const int32_t* ind, const Workspace& ws, uint32_t* out, const SchedParams& sp,
                       cudaStream_t stream) {
  constexpr int kMaxDev = 64;
  static int blocks_per_sm[kMaxDev] = {};  // 0 = not configured on that device yet
  const size_t smem = sizeof(CountSmem);
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  if (blocks_per_sm[dev] == 0) {
    TC_CUDA_TRY(cudaFuncSetAttribute(k_count<PV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int b = 0;
    TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_count<PV>, kThreads, smem));
    blocks_per_sm[dev] = std::max(1, b);
  }
  const int bps = sp.blocks_per_sm > 0 ? std::min(sp.blocks_per_sm, blocks_per_sm[dev]) : blocks_per_sm[dev];
  const int grid = device_info().sms * bps;
#ifdef TC_DEBUG_PROGRESS
  if (tc_dbg_progress_host_dev) cudaMemsetAsync(tc_dbg_progress_host_dev, 0, tc_dbg_progress_bytes, stream);
#endif
  k_count<PV><<<grid, kThreads, smem, stream>>>(n, ind, ws.degv, ws.dplus, ws.offp, ws.indp, ws.large, ws.medium, out,
                                                ws.st, sp);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

// Grid of a persistent kernel: every CTA resident at once (occupancy looked up once per device).
template <auto kernel>
tc_status resident_grid(int threads, int* grid) {
  constexpr int kMaxDev = 64;
  static int per_sm[kMaxDev] = {};
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  if (per_sm[dev] == 0) {
    int b = 0;
    TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0));
    per_sm[dev] = std::max(1, b);
  }
  *grid = device_info().sms * per_sm[dev];
  return TC_OK;
}

template <class View>
tc_status orient(const View& view, int32_t n, Workspace& ws, const SchedParams& sp, bool write, cudaStream_t stream) {
  k_find_hubs<View><<<hubs_grid(n), 256, 0, stream>>>(view, n, ws.dplus, ws.offp, ws.degv, ws.hub_u, ws.hub_base,
                                                      ws.hub_done, ws.chunk_hub, ws.hub_cap, ws.chunk_cap, ws.st);
  TC_CUDA_TRY(cudaGetLastError());
  int grid = 0;
  if (write) TC_TRY((resident_grid<k_orient<View, true>>(256, &grid)));
  else TC_TRY((resident_grid<k_orient<View, false>>(256, &grid)));
  if (write)
    k_orient<View, true><<<grid, 256, 0, stream>>>(view, n, ws.dplus, ws.offp, ws.degv, ws.indp, ws.e_cap,
                                                   ws.hub_u, ws.hub_base, ws.hub_cnt, ws.hub_done, ws.chunk_hub,
                                                   ws.hub_cap, ws.chunk_cap, ws.st);
  else
    k_orient<View, false><<<grid, 256, 0, stream>>>(view, n, ws.dplus, ws.offp, ws.degv, ws.indp, ws.e_cap,
                                                    ws.hub_u, ws.hub_base, ws.hub_cnt, ws.hub_done, ws.chunk_hub,
                                                    ws.hub_cap, ws.chunk_cap, ws.st);
  TC_CUDA_TRY(cudaGetLastError());
  if (write) {
    if (sp.nshards > 1) {
      // this count's range of centres: predicted work per centre, its prefix, the range
      if (!ws.shard_cost || ws.shard_cap < (int64_t)n + 1)
        return fail(TC_ERR_STATE, "sharded count without its shard workspace");
      k_shard_cost<View><<<orient_grid(n), 256, 0, stream>>>(view, n, ws.dplus, ws.shard_cost);
      TC_CUDA_TRY(cudaGetLastError());
      TC_TRY(scan_counts(ws.shard_cost, n, ws.shard_prefix, ws.shard_tiles, stream));
      k_shard_bounds<<<1, 32, 0, stream>>>(ws.shard_prefix, n, sp.shard, sp.nshards, ws.st);
      TC_CUDA_TRY(cudaGetLastError());
    }
    // the count's work queues (only a count reads them)
    k_push_items<<<hubs_grid(n), 256, 0, stream>>>(n, ws.dplus, ws.degv, ws.medium, ws.item_cap, ws.st, sp.warp_max);
    TC_CUDA_TRY(cudaGetLastError());
    k_fill_items<<<hubs_grid(n), 256, 0, stream>>>(n, ws.dplus, ws.degv, ws.large, ws.item_cap, ws.st, sp.warp_max);
    TC_CUDA_TRY(cudaGetLastError());
  }
  return TC_OK;
}

}  // namespace

int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

tc_status scan_counts(const int32_t* in, int64_t n, int64_t* out, int64_t* tile_sums, cudaStream_t stream) {
  const int64_t nt = scan_tiles(n);
  if (nt == 0) {
    TC_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t), stream));
    return TC_OK;
  }
  k_scan_tile_sums<<<(unsigned)nt, kScanThreads, 0, stream>>>(in, n, tile_sums);
  k_scan_tile_prefix<<<1, 1024, 0, stream>>>(tile_sums, nt);
  k_scan_tiles<<<(unsigned)nt, kScanThreads, 0, stream>>>(in, n, tile_sums, out, nt);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

SchedParams to_params(const tc_sched* s) {
  tc_sched d;
  if (!s) {
    tc_sched_default(&d);
    s = &d;
  }
  SchedParams p;
  p.warp_max = std::min(kWarpTierMax, std::max(2, s->warp_max_deg));
  p.search_ratio_x16 = std::max(0, s->search_ratio_x16);
  p.use_table = s->use_table ? 1 : 0;
  p.chunk = std::max(32, (s->chunk + 31) / 32 * 32);
  p.blocks_per_sm = std::max(0, s->blocks_per_sm);
  p.nshards = std::max(1, s->nshards);
  p.shard = std::min(std::max(0, s->shard), p.nshards - 1);
  p.cell_filter = s->cell_filter < -2 ? -1 : s->cell_filter;
  p.lane_max = std::min(64, std::max(0, s->lane_max_deg));
  p.packed_max = std::max(0, s->packed_max_deg);
  p.hub_min = std::max(0, s->stream_hub_min);
  memcpy(p.table, s->table, sizeof(p.table));
  return p;
}

template <class View>
tc_status static_count(const View& view, int32_t n, int64_t m, Workspace& ws, int pv_mode, int32_t* per_vertex,
                       int64_t* triangles_dev, const SchedParams& sp, cudaStream_t stream) {
  if (sp.nshards > 1 && n > 0) TC_TRY(ws.ensure_shards(n));
  TC_CUDA_TRY(cudaMemsetAsync(ws.st, 0, sizeof(DevStatus), stream));
  if (pv_mode != TC_PV_NONE && n > 0)
    TC_CUDA_TRY(cudaMemsetAsync(per_vertex, 0, (pv_mode == TC_PV_HANDLE64 ? 8 : 4) * (size_t)n, stream));
  if (n > 0) {
    prof_mark(0, stream);
    TC_TRY(orient(view, n, ws, sp, true, stream));
    prof_mark(1, stream);
    uint32_t* out = reinterpret_cast<uint32_t*>(per_vertex);
    switch (pv_mode) {
      case TC_PV_NONE: TC_TRY(launch_count<TC_PV_NONE>(n, view.ind, ws, out, sp, stream)); break;
      case TC_PV_HANDLE: TC_TRY(launch_count<TC_PV_HANDLE>(n, view.ind, ws, out, sp, stream)); break;
      case TC_PV_CSR: TC_TRY(launch_count<TC_PV_CSR>(n, view.ind, ws, out, sp, stream)); break;
      case TC_PV_HANDLE64: TC_TRY(launch_count<TC_PV_HANDLE64>(n, view.ind, ws, out, sp, stream)); break;
      default: return fail(TC_ERR_INVALID_ARG, "unknown per-vertex mode %d", pv_mode);
    }
    prof_mark(2, stream);
    // k_find_hubs, k_orient, k_push_items, k_fill_items, k_count (+ k_shard_cost, three scan
    // kernels and k_shard_bounds when sharded)
    prof_launches(sp.nshards > 1 ? 10 : 5);
  }
  (void)m;
  if (triangles_dev)
    TC_CUDA_TRY(cudaMemcpyAsync(triangles_dev, &ws.st->triangles, sizeof(int64_t), cudaMemcpyDeviceToDevice, stream));
  return TC_OK;
}

template tc_status static_count<Csr32View>(const Csr32View&, int32_t, int64_t, Workspace&, int, int32_t*, int64_t*,
                                           const SchedParams&, cudaStream_t);
template tc_status static_count<Csr64View>(const Csr64View&, int32_t, int64_t, Workspace&, int, int32_t*, int64_t*,
                                           const SchedParams&, cudaStream_t);
template tc_status static_count<SlackView>(const SlackView&, int32_t, int64_t, Workspace&, int, int32_t*, int64_t*,
                                           const SchedParams&, cudaStream_t);

tc_status read_info(const Workspace& ws, cudaStream_t stream, tc_count_info* info) {
  DevStatus h;
  TC_CUDA_TRY(cudaMemcpyAsync(&h, ws.st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
  TC_CUDA_TRY(cudaStreamSynchronize(stream));
  info->triangles = (int64_t)h.triangles;
  info->edges_intersected = (int64_t)h.edges_intersected;
  info->oriented_work = (int64_t)h.oriented_work;
  info->max_out_degree = (int32_t)h.max_dplus;
  info->shard_lo = h.sharded ? (int32_t)h.shard_lo : 0;
  info->shard_hi = h.sharded ? (int32_t)h.shard_hi : -1;
  info->shard_work = (int64_t)h.shard_work;
  info->total_work = (int64_t)h.total_work;
  if (h.bad_flags & (kBadRange | kBadOrder | kBadSelfLoop)) {
    info->status = TC_ERR_BAD_GRAPH;
    return fail(TC_ERR_BAD_GRAPH, "graph check failed:%s%s%s", (h.bad_flags & kBadRange) ? " id out of range" : "",
                (h.bad_flags & kBadOrder) ? " list not strictly ascending" : "",
                (h.bad_flags & kBadSelfLoop) ? " self-loop" : "");
  }
  if (h.bad_flags & kBadCapacity) {
    info->status = TC_ERR_CAPACITY;
    return fail(TC_ERR_CAPACITY, "oriented graph exceeded its workspace");
  }
  if (h.bad_flags & kBadTimeout) {
    info->status = TC_ERR_TIMEOUT;
    return fail(TC_ERR_TIMEOUT, "a staged copy of the count kernel did not land in time; the count is incomplete");
  }
  if (h.sym_checksum != 0) {
    info->status = TC_ERR_NOT_SYMMETRIC;
    return fail(TC_ERR_NOT_SYMMETRIC, "adjacency is not symmetric");
  }
  info->status = TC_OK;
  return TC_OK;
}

namespace {
// Warp per source vertex: per degree-cell sums over its oriented edges, in shared memory, then
// one atomic per touched cell per CTA.
__global__ void __launch_bounds__(256) k_cell_stats(const int32_t n, const int32_t* __restrict__ dplus,
                                                    const int64_t* __restrict__ offp, const int32_t* __restrict__ indp,
                                                    double* __restrict__ out) {
  __shared__ double acc[256 * 4];
  for (int i = threadIdx.x; i < 256 * 4; i += blockDim.x) acc[i] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t uu = gw; uu < n; uu += nw) {
    const int32_t du = dplus[uu];
    const int64_t s = offp[uu];
    for (int32_t k = lane; k < du; k += 32) {
      // the cell the count files the edge under: (centre's out-degree, the other endpoint's)
      const int32_t dv = dplus[indp[s + k]];
      const int32_t a = max(du, dv), b = min(du, dv);
      const int c = log2_cell(a) * 16 + log2_cell(b);
      atomicAdd(&acc[4 * c + 0], 1.0);
      atomicAdd(&acc[4 * c + 1], log2(1.0 + a));
      atomicAdd(&acc[4 * c + 2], log2(1.0 + b));
      atomicAdd(&acc[4 * c + 3], (double)b / (double)max(a, 1));
    }
  }
  __syncwarp();
  __syncthreads();
  for (int i = threadIdx.x; i < 256 * 4; i += blockDim.x)
    if (acc[i] != 0.0) atomicAdd(&out[i], acc[i]);
}
}  // namespace

tc_status cell_stats(int32_t n, Workspace& ws, double* out_host, cudaStream_t stream) {
  double* d = nullptr;
  TC_CUDA_TRY(::tc::dev_malloc(&d, sizeof(double) * 1024));
  cudaMemsetAsync(d, 0, sizeof(double) * 1024, stream);
  if (n > 0) k_cell_stats<<<orient_grid(n), 256, 0, stream>>>(n, ws.dplus, ws.offp, ws.indp, d);
  cudaError_t e = cudaMemcpyAsync(out_host, d, sizeof(double) * 1024, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, "cell stats: %s", cudaGetErrorString(e));
  return TC_OK;
}

template <class View>
tc_status validate_view(const View& view, int32_t n, Workspace& ws, cudaStream_t stream) {
  TC_CUDA_TRY(cudaMemsetAsync(ws.st, 0, sizeof(DevStatus), stream));
  if (n > 0) TC_TRY(orient(view, n, ws, to_params(nullptr), false, stream));
  return TC_OK;
}

template tc_status validate_view<SlackView>(const SlackView&, int32_t, Workspace&, cudaStream_t);
template tc_status validate_view<Csr64View>(const Csr64View&, int32_t, Workspace&, cudaStream_t);

}  // namespace tc

#ifdef TC_DEBUG_PROGRESS
extern "C" {
volatile int tc_dbg_host_stage = 0;
void* tc_dbg_progress_host_dev = nullptr;
size_t tc_dbg_progress_bytes = 0;
int tc_debug_get_stage(void) { return tc_dbg_host_stage; }
int tc_debug_set_progress(void* dev_ptr, size_t bytes, void* kern_dev_ptr) {
  unsigned long long* p = (unsigned long long*)dev_ptr;
  unsigned long long* k = (unsigned long long*)kern_dev_ptr;
  tc_dbg_progress_host_dev = dev_ptr;
  tc_dbg_progress_bytes = bytes;
  int e = (int)cudaMemcpyToSymbol(tc::tc_dbg_progress, &p, sizeof(p));
  if (e) return e;
  return (int)cudaMemcpyToSymbol(tc::tc_dbg_kern, &k, sizeof(k));
}
}
#endif
