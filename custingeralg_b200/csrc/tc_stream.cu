// Streaming triangle counting: batch preparation, structural updates of the slack-managed
// adjacency and the triangle delta of a batch (sm_100a).
//
// Replaces the reference's three streaming kernels devicecuStingerNewTriangles,
// deviceBUThreeTriangles and deviceBUTwoCUOneTriangles (src/streaming_triangle_counting/
// cct_upd.cu:231-410), whose inclusion-exclusion nets +2 per vertex of every new triangle on a
// symmetric batch (K1 counts a triangle with k new edges k times, K2 and K3 correct the
// overcount). Here a triangle is attributed once, to the smallest of its changed edges in the
// (min id, max id) order: k_delta intersects N(x) and N(y) for each changed edge {x, y} and keeps
// a common neighbour w unless (x, w) or (y, w) is a changed edge with a smaller key. Whether an
// edge is changed comes either from a per-slot mark array parallel to the adjacency pool
// (tc_apply_batch) or from a lookup in the sorted batch (the cuStinger-style path).
//
// Per changed edge the warp intersects the two full lists with a strategy chosen by their
// lengths: binary search of the shorter list's entries into the longer ("search", for skewed
// pairs), a partitioned merge in which each lane owns a contiguous slice of the shorter list and
// merges it against the longer one from a binary-searched start ("merge", for balanced pairs), or,
// where the strategy table asks for it, the longer list staged into shared memory piece by piece
// with cp.async and searched there ("stage").
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "tc_graph.cuh"

namespace tc {

namespace {

constexpr int kThreads = 256;
constexpr uint64_t kSentinel = ~0ull;
constexpr int kLongList = 2048;  // lists longer than this are rewritten by a whole CTA
// Tile shape of the delta count (defaults; the pipeline's autotuner picks per batch-size bin):
constexpr int kDeltaSplit = 2048;   // intersections whose shorter list is longer are split ...
constexpr int kDeltaChunk = 1024;   // ... into items of this many entries of the shorter list
constexpr int64_t kDeltaItems = 1 << 20;  // capacity of the split-item queue
constexpr unsigned long long kNoItem = ~0ull;
constexpr int kGrab = 4;  // changed edges a warp takes per grab from the delta kernel's queue
// Bound of the persistent delta kernel's waits for queued split items (a wait that runs out
// reports kErrTimeout and the warp leaves the item pass).
constexpr unsigned long long kSpinNs = 2000000000ull;  // 2 s
constexpr unsigned kSpinMaxIters = 1u << 24;

enum : unsigned { kErrRange = 1u, kErrPool = 2u, kErrTimeout = 4u, kErrScratch = 8u };
// first_del[v] between batches: no deletion marked in v's list (0x7f7f7f7f, a byte memset)
constexpr int32_t kNoDel = 0x7f7f7f7f;
constexpr unsigned long long kNoLongItem = ~0ull;

struct BatchStatus {
  unsigned long long n_uniq;      // unique undirected edges
  unsigned long long n_del;       // effective deletions
  unsigned long long n_ins;       // effective insertions
  unsigned long long n_dir;       // directed insert entries (2 n_ins)
  unsigned long long n_runs;      // affected source vertices of insertions
  unsigned long long demand;      // pool slots relocations may take
  unsigned long long tri_removed;
  unsigned long long tri_added;
  unsigned long long pool_top;    // device copy of the bump pointer
  unsigned long long dir_added;   // directed entries inserted (cuStinger path)
  unsigned long long dir_removed; // directed entries deleted (cuStinger path)
  unsigned long long not_fitting;
  unsigned long long n_long;      // insertion runs whose list is long (k_long_plan)
  unsigned long long long_scr;    // scratch entries and work items of the long-list insertion
  unsigned long long long_items;
  unsigned long long n_cmp;       // long lists compacted, their scratch entries and work items
  unsigned long long cmp_scr;
  unsigned long long cmp_items;
  unsigned long long n_split[2];  // split-intersection items queued (deletions, insertions)
  unsigned long long delta_bytes; // algorithmic bytes of the batch's intersections (4(deg x + deg y) + 8 each)
  unsigned int entry_done[2];     // warps of the persistent delta kernel done with the entry pass
  unsigned int err;
  unsigned int pad;
  unsigned long long n_hubs[2];   // hub groups of the delta count (deletions, insertions)
  unsigned long long hub_total[2];  // changed edges placed in hub groups
  unsigned long long hub_q[2];    // work-queue heads of the hub kernel
  unsigned long long hub_items[2];  // hub work items queued
  unsigned long long e_next[2];   // work-queue heads of the delta kernel's entry and item passes
  unsigned long long i_next[2];
};

__device__ __forceinline__ uint64_t ekey(int32_t a, int32_t b) {
  const uint32_t lo = (uint32_t)min(a, b), hi = (uint32_t)max(a, b);
  return ((uint64_t)lo << 32) | hi;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

// First index in [lo, hi) of list with list[i] >= key.
__device__ __forceinline__ int64_t lower_bound(const int32_t* __restrict__ list, int64_t lo, int64_t hi, int32_t key) {
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(list + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// First index of the ascending list lst[0 .. len) whose entry is >= key, found by the warp: 32
// evenly spaced samples per round (one load each lane), so a list of up to 32^r entries takes r
// rounds. Every lane returns the same index.
__device__ __forceinline__ int32_t warp_lower_bound(const int32_t* __restrict__ lst, int32_t len, int32_t key) {
  const int lane = threadIdx.x & 31;
  int32_t lo = 0, hi = len;  // the answer lies in [lo, hi]
  while (hi - lo > 32) {
    const int32_t step = (hi - lo + 31) / 32;
    const int32_t p = lo + lane * step;
    const int32_t v = p < hi ? lst[p] : INT32_MAX;
    const int c = __popc(__ballot_sync(kFull, v < key));  // the samples below key are a prefix
    const int32_t nlo = c > 0 ? lo + (c - 1) * step + 1 : lo;
    hi = c < 32 ? min(hi, lo + c * step) : hi;
    lo = nlo;
  }
  const int32_t p = lo + lane;
  const int32_t v = p < hi ? lst[p] : INT32_MAX;
  return lo + __popc(__ballot_sync(kFull, v < key));
}

// Asynchronous 4-byte copy from global to shared memory (cp.async, no register round trip); the
// copies of a thread complete at cp_async_wait_all.
__device__ __forceinline__ void cp_async4(int32_t* smem_dst, const int32_t* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// GPU-scope release store and acquire loads (publication of work items between CTAs).
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

int grid_for(int64_t items, int per_block) {
  const int64_t want = std::max<int64_t>(1, (items + per_block - 1) / per_block);
  return (int)std::min<int64_t>(want, (int64_t)device_info().sms * 16);
}

// ---- batch preparation (canonical undirected updates) --------------------------------------

// key = (min << (L+1)) | (max << 1) | is_insert; self-loops and bad ids become the sentinel.
__global__ void k_make_keys(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                            const uint8_t* __restrict__ is_del, const int64_t b, const int32_t n, const int L,
                            uint64_t* __restrict__ keys, BatchStatus* __restrict__ st) {
  const uint64_t sent = (1ull << (2 * L + 1)) - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s = src[i], d = dst[i];
    uint64_t k = sent;
    if (s < 0 || s >= n || d < 0 || d >= n) {
      atomicOr(&st->err, kErrRange);
    } else if (s != d) {
      const uint64_t lo = (uint64_t)min(s, d), hi = (uint64_t)max(s, d);
      k = (lo << (L + 1)) | (hi << 1) | (uint64_t)((is_del && is_del[i]) ? 0 : 1);
    }
    keys[i] = k;
  }
}

__global__ void k_run_heads(const uint64_t* __restrict__ keys, const int64_t b, const uint64_t sent,
                            int32_t* __restrict__ head) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    head[i] = (k != sent) && (i == 0 || (keys[i - 1] >> 1) != (k >> 1));
  }
}

// Each unique undirected edge: classify against the graph and append to the deletion or the
// insertion list. A deletion records the slots of the edge in both lists.
__global__ void k_classify(const SlackView g, const uint64_t* __restrict__ keys, const int64_t b, const int L,
                           const int32_t* __restrict__ head, int4* __restrict__ dlist, int2* __restrict__ ilist,
                           uint64_t* __restrict__ dirkeys, BatchStatus* __restrict__ st) {
  const uint64_t maxmask = (1ull << L) - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const uint64_t e = keys[i] >> 1;
    int64_t j = i;
    while (j + 1 < b && (keys[j + 1] >> 1) == e) ++j;
    const bool del_any = (keys[i] & 1ull) == 0;  // deletions sort before insertions of the same edge
    const bool ins_any = (keys[j] & 1ull) == 1;
    const int32_t x = (int32_t)(e >> L), y = (int32_t)(e & maxmask);
    atomicAdd(&st->n_uniq, 1ull);
    // presence: search the shorter list
    const int32_t lx = g.len(x), ly = g.len(y);
    const int64_t sx = g.start(x), sy = g.start(y);
    int64_t px = -1, py = -1;
    if (lx <= ly) {
      const int64_t p = lower_bound(g.ind, sx, sx + lx, y);
      if (p < sx + lx && g.ind[p] == y) px = p - sx;
    } else {
      const int64_t p = lower_bound(g.ind, sy, sy + ly, x);
      if (p < sy + ly && g.ind[p] == x) py = p - sy;
    }
    const bool present = px >= 0 || py >= 0;
    if (del_any && !ins_any && present) {
      if (px < 0) px = lower_bound(g.ind, sx, sx + lx, y) - sx;
      if (py < 0) py = lower_bound(g.ind, sy, sy + ly, x) - sy;
      const unsigned long long at = atomicAdd(&st->n_del, 1ull);
      dlist[at] = make_int4(x, y, (int32_t)px, (int32_t)py);
    } else if (ins_any && !present) {
      const unsigned long long at = atomicAdd(&st->n_ins, 1ull);
      ilist[at] = make_int2(x, y);
      dirkeys[2 * at] = ((uint64_t)(uint32_t)x << 32) | (uint32_t)y;
      dirkeys[2 * at + 1] = ((uint64_t)(uint32_t)y << 32) | (uint32_t)x;
    }
  }
}

// ---- insertion planning / application ------------------------------------------------------

// Heads of source-vertex runs in the sorted directed entries, and the pool slots the lists that
// must move could take (computed on the pre-deletion lengths, an upper bound).
// A run whose list will be long (used + new > kLongList) is stored as -1 - start and also listed
// (start, length) in long_runs / long_cnt for the long-list insertion; the warp kernel skips it.
__global__ void k_dir_runs(const uint64_t* __restrict__ dk, const int64_t nd_cap, const int32_t* __restrict__ used,
                           const int32_t* __restrict__ cap, const int32_t slack_q10, int32_t* __restrict__ run_start,
                           int32_t* __restrict__ long_runs, int32_t* __restrict__ long_cnt,
                           BatchStatus* __restrict__ st) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nd_cap; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = dk[i];
    if (k == kSentinel) continue;
    const uint32_t v = (uint32_t)(k >> 32);
    if (i > 0 && (uint32_t)(dk[i - 1] >> 32) == v) continue;
    int64_t j = i;
    while (j + 1 < nd_cap && dk[j + 1] != kSentinel && (uint32_t)(dk[j + 1] >> 32) == v) ++j;
    const int32_t c = (int32_t)(j - i + 1);
    const unsigned long long r = atomicAdd(&st->n_runs, 1ull);
    const int32_t need = used[v] + c;
    if (need > kLongList) {
      run_start[r] = -1 - (int32_t)i;
      const unsigned long long q = atomicAdd(&st->n_long, 1ull);
      long_runs[q] = (int32_t)i;
      long_cnt[q] = c;
    } else {
      run_start[r] = (int32_t)i;
    }
    if (need > cap[v]) atomicAdd(&st->demand, (unsigned long long)slack_capacity(need, max(slack_q10, 256)));
  }
}

// One warp per affected source vertex: merge its sorted new neighbours into its list, in place
// (backwards) when the capacity allows, else into a fresh block at the pool top. New slots are
// marked (mark = 1) when `mark` is given; their absolute slots go to slot[].
__global__ void k_insert_runs(const uint64_t* __restrict__ dk, const int64_t nd_cap, const int32_t* __restrict__ run_start,
                              int64_t* __restrict__ start, int32_t* __restrict__ used, int32_t* __restrict__ cap,
                              int32_t* __restrict__ pool, const int64_t pool_cap, uint8_t* __restrict__ mark,
                              int64_t* __restrict__ slot, unsigned long long* __restrict__ pool_top,
                              const int32_t slack_q10, BatchStatus* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t nruns = (int64_t)st->n_runs;
  for (int64_t r = gw; r < nruns; r += nw) {
    const int64_t i0 = run_start[r];
    if (i0 < 0) continue;  // a long list: k_long_plan / k_long_stage / k_long_write
    const int32_t v = (int32_t)(dk[i0] >> 32);
    int64_t i1 = i0;  // run end (exclusive), found cooperatively
    {
      int64_t k = i0 + lane;
      while (true) {
        const bool same = k < nd_cap && dk[k] != kSentinel && (int32_t)(dk[k] >> 32) == v;
        __syncwarp();
        const unsigned m = __ballot_sync(kFull, same);
        if (m != kFull) {
          i1 = k - lane + __ffs(~m) - 1;
          break;
        }
        k += 32;
      }
      i1 = __shfl_sync(kFull, i1, 0);
    }
    const int32_t c = (int32_t)(i1 - i0);
    const int32_t a = used[v];
    const int64_t s_old = start[v];
    int64_t s_new = s_old;
    bool moved = false;
    if (a + c > cap[v]) {
      const int32_t nc = slack_capacity(a + c, max(slack_q10, 256));
      unsigned long long at = 0;
      if (lane == 0) at = atomicAdd(pool_top, (unsigned long long)nc);
      __syncwarp();
      at = __shfl_sync(kFull, at, 0);
      __syncwarp();
      if ((int64_t)at + nc > pool_cap) {
        if (lane == 0) atomicOr(&st->err, kErrPool);
        for (int64_t j = i0 + lane; j < i1; j += 32) slot[j] = -1;  // nothing to clear later
        continue;  // cannot happen when the host sized the pool from the demand pass
      }
      s_new = (int64_t)at;
      moved = true;
      if (lane == 0) {
        cap[v] = nc;
        atomicAdd(&st->not_fitting, (unsigned long long)c);
      }
    }
    const int32_t* A = pool + s_old;
    // New entries first, while A is intact: final position j + #(old < B[j]) (relative). The
    // first five levels of each search come from 32 evenly spaced samples of A held in the lanes.
    int32_t first_new = a;  // old entries below the smallest new entry keep their slots
    {
      const int32_t step = (a + 31) / 32;
      const int32_t smp = lane * step < a ? A[lane * step] : INT32_MAX;
      const int32_t s31 = __shfl_sync(kFull, smp, 31);
      for (int64_t jb = i0; jb < i1; jb += 32) {
        const int64_t j = jb + lane;
        const bool act = j < i1;
        const int32_t val = act ? (int32_t)(uint32_t)dk[j] : INT32_MAX;
        int pos = 0;  // samples below val (they ascend with the lane)
#pragma unroll
        for (int st = 16; st > 0; st >>= 1)
          if (__shfl_sync(kFull, smp, pos + st - 1) < val) pos += st;
        if (pos == 31 && s31 < val) pos = 32;
        int32_t lo = pos > 0 ? (pos - 1) * step + 1 : 0;
        int32_t hi = pos < 32 ? min(pos * step, a) : a;
        if (act) {
          while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (A[mid] < val) lo = mid + 1;
            else hi = mid;
          }
          slot[j] = (j - i0) + lo;
          if (j == i0) first_new = lo;
        }
        __syncwarp();
      }
    }
    __syncwarp();
    // In place, old entries below the first new entry do not move; relocated, all of them do.
    const int32_t keep_below = moved ? 0 : __shfl_sync(kFull, first_new, 0);
    // Old entries: final position i + #(new < A[i]); backwards in chunks so that, in place, no
    // unread entry is overwritten (targets never precede sources). Each chunk's entries are read
    // one chunk ahead: the writes of a chunk go to slots at or above its own.
    const int32_t low = (keep_below / 32) * 32;
    int32_t base = a > 0 ? ((a - 1) / 32) * 32 : -1;
    int32_t ahead = (base >= low && base + lane < a && base + lane >= keep_below) ? A[base + lane] : 0;
    for (; base >= low; base -= 32) {
      const int32_t i = base + lane;
      const bool act = i < a && i >= keep_below;
      const int32_t val = ahead;
      const int32_t inext = i - 32;
      ahead = (base - 32 >= low && inext >= keep_below) ? A[inext] : 0;
      int64_t pos = 0;
      if (act) {
        int64_t lo = i0, hi = i1;
        while (lo < hi) {
          const int64_t mid = (lo + hi) >> 1;
          if ((int32_t)(uint32_t)dk[mid] < val) lo = mid + 1;
          else hi = mid;
        }
        pos = i + (lo - i0);
      }
      __syncwarp();
      if (act) {
        pool[s_new + pos] = val;
        if (mark) mark[s_new + pos] = 0;
      }
      __syncwarp();
    }
    // New entries into the holes.
    for (int64_t j = i0 + lane; j < i1; j += 32) {
      const int64_t pos = s_new + slot[j];
      pool[pos] = (int32_t)(uint32_t)dk[j];
      if (mark) mark[pos] = 1;
      slot[j] = pos;
    }
    __syncwarp();
    if (lane == 0) {
      used[v] = a + c;
      if (moved) start[v] = s_new;
      atomicAdd(&st->dir_added, (unsigned long long)c);
    }
  }
}

// Clear the marks of the inserted slots: n_host entries, or 2 * (*n_dev) when n_dev is given.
__global__ void k_clear_slots(const int64_t* __restrict__ slot, const int64_t n_host,
                              const unsigned long long* __restrict__ n_dev, uint8_t* __restrict__ mark) {
  const int64_t n = n_dev ? 2 * (int64_t)(*n_dev) : n_host;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = slot[i];
    if (s >= 0) mark[s] = 0;
  }
}

// ---- deletion -------------------------------------------------------------------------------

// Mark the slots of the batch's deletions and keep each list's smallest marked slot (the
// compaction leaves the entries below it in place).
__global__ void k_mark_deletions(const int4* __restrict__ dlist, const BatchStatus* __restrict__ st,
                                 const int64_t* __restrict__ start, uint8_t* __restrict__ mark,
                                 int32_t* __restrict__ first_del) {
  const int64_t nd = (int64_t)st->n_del;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += (int64_t)gridDim.x * blockDim.x) {
    const int4 d = dlist[i];
    mark[start[d.x] + d.z] = 1;
    mark[start[d.y] + d.w] = 1;
    atomicMin(&first_del[d.x], d.z);
    atomicMin(&first_del[d.y], d.w);
  }
}

// Remove marked slots from the lists of the vertices in vlist (each vertex once: the first warp
// to claim it with this epoch compacts it), then clear the marks of the old range. The entries
// below the list's first marked slot (first_del, reset here to kNoDel) stay where they are.
__global__ void k_compact_marked(const int32_t* __restrict__ vlist, const int64_t nv_list, const int stride,
                                 const unsigned long long* __restrict__ nv_dev, const int64_t* __restrict__ start,
                                 int32_t* __restrict__ used, int32_t* __restrict__ pool, uint8_t* __restrict__ mark,
                                 unsigned* __restrict__ claim, const unsigned* __restrict__ epoch_dev,
                                 int32_t* __restrict__ first_del, BatchStatus* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  const unsigned epoch = *epoch_dev;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t cnt = nv_dev ? (int64_t)(*nv_dev) * stride : nv_list;
  const unsigned lt = (1u << lane) - 1u;
  for (int64_t k = gw; k < cnt; k += nw) {
    const int32_t v = vlist[k];
    if (used[v] > kLongList) continue;  // a long list: k_cmp_plan / stage / prefix / write
    unsigned old = 0;
    if (lane == 0) old = atomicMax(&claim[v], epoch);
    __syncwarp();
    old = __shfl_sync(kFull, old, 0);
    if (old >= epoch) continue;
    const int64_t s = start[v];
    const int32_t a = used[v];
    const int32_t f = min(first_del[v], a);
    __syncwarp();
    if (lane == 0) first_del[v] = kNoDel;
    int32_t wp = f;
    for (int32_t base = f; base < a; base += 32) {
      const int32_t i = base + lane;
      int32_t val = 0;
      bool keep = false;
      if (i < a) {
        val = pool[s + i];
        keep = mark[s + i] == 0;
      }
      __syncwarp();
      const unsigned m = __ballot_sync(kFull, keep);
      __syncwarp();
      if (keep) pool[s + wp + __popc(m & lt)] = val;
      wp += __popc(m);
      __syncwarp();
    }
    for (int32_t i = f + lane; i < a; i += 32) mark[s + i] = 0;
    if (lane == 0) {
      used[v] = wp;
      atomicAdd(&st->dir_removed, (unsigned long long)(a - wp));
    }
  }
}


// Insertion into long lists (more than kLongList entries after the batch), in three launches
// over all of the batch's long runs at once:
//   k_long_plan   one thread per run: relocation (when the list outgrows its capacity) or the
//                 in-place merge's first moving entry (the first new entry's slot), the list's
//                 new length, a range of the scratch buffer and work items of kLongChunk entries;
//   k_long_stage  one CTA per item: each moving old entry and each new entry computes its place
//                 in the merged suffix (an old entry shifts by the number of new entries below it,
//                 a new entry lands after the old entries below it) and writes there in scratch;
//   k_long_write  one CTA per item: the merged suffix back into the list, with the new entries'
//                 marks.
// The launch boundary between staging and writing takes the place of an in-place merge's block
// barriers: every source is read before any target is written, so a hub list of 10^5 entries is
// spread over many CTAs instead of being one CTA's chain of steps.
constexpr int kLongChunk = 4096;

struct LongPlan {
  int64_t s_old;   // list start before the batch
  int64_t s_new;   // list start after it (s_old unless relocated)
  int64_t soff;    // the run's range in the scratch buffer
  int32_t a;       // entries before the batch
  int32_t c;       // new entries
  int32_t first;   // first moving entry (0 when relocated)
  int32_t len;     // entries staged: a - first + c (0 = nothing to do)
  int32_t i0;      // the run's first entry in the sorted directed keys
  int32_t pad;
};

__global__ void __launch_bounds__(kThreads) k_long_plan(
    const uint64_t* __restrict__ dk, const int32_t* __restrict__ long_runs, const int32_t* __restrict__ long_cnt,
    int64_t* __restrict__ start, int32_t* __restrict__ used, int32_t* __restrict__ cap,
    const int32_t* __restrict__ pool, const int64_t pool_cap, int64_t* __restrict__ slot,
    unsigned long long* __restrict__ pool_top, const int32_t slack_q10, LongPlan* __restrict__ plan,
    unsigned long long* __restrict__ items, const int64_t item_cap, const int64_t scr_cap,
    BatchStatus* __restrict__ st) {
  const int64_t nlong = (int64_t)st->n_long;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nlong; r += (int64_t)gridDim.x * blockDim.x) {
    LongPlan P;
    P.i0 = long_runs[r];
    P.c = long_cnt[r];
    P.pad = 0;
    const int32_t v = (int32_t)(dk[P.i0] >> 32);
    P.a = used[v];
    P.s_old = start[v];
    P.s_new = P.s_old;
    P.len = 0;
    P.soff = 0;
    P.first = 0;
    bool ok = true;
    if (P.a + P.c > cap[v]) {
      const int32_t nc = slack_capacity(P.a + P.c, max(slack_q10, 256));
      const unsigned long long at = atomicAdd(pool_top, (unsigned long long)nc);
      if ((int64_t)at + nc > pool_cap) {
        atomicOr(&st->err, kErrPool);
        ok = false;
      } else {
        P.s_new = (int64_t)at;
        start[v] = P.s_new;
        cap[v] = nc;
        atomicAdd(&st->not_fitting, (unsigned long long)P.c);
      }
    } else {
      P.first = (int32_t)(lower_bound(pool, P.s_old, P.s_old + P.a, (int32_t)(uint32_t)dk[P.i0]) - P.s_old);
    }
    if (ok) {
      P.len = P.a - P.first + P.c;
      const int32_t nch = (P.len + kLongChunk - 1) / kLongChunk;
      const unsigned long long so = atomicAdd(&st->long_scr, (unsigned long long)P.len);
      const unsigned long long ib = atomicAdd(&st->long_items, (unsigned long long)nch);
      if ((int64_t)(so + P.len) > scr_cap || (int64_t)(ib + nch) > item_cap) {
        atomicOr(&st->err, kErrScratch);  // unreachable while the scratch follows the pool's size
        ok = false;
        for (int32_t j = 0; j < nch && (int64_t)(ib + j) < item_cap; ++j) items[ib + j] = kNoLongItem;
      } else {
        P.soff = (int64_t)so;
        for (int32_t j = 0; j < nch; ++j) items[ib + j] = ((unsigned long long)r << 32) | (unsigned)j;
        used[v] = P.a + P.c;
        atomicAdd(&st->dir_added, (unsigned long long)P.c);
      }
    }
    if (!ok) {
      P.len = 0;
      for (int32_t j = 0; j < P.c; ++j) slot[P.i0 + j] = -1;
    }
    plan[r] = P;
  }
}

__global__ void __launch_bounds__(kThreads) k_long_stage(
    const uint64_t* __restrict__ dk, const int32_t* __restrict__ pool, const LongPlan* __restrict__ plan,
    const unsigned long long* __restrict__ items, const int64_t item_cap, int32_t* __restrict__ scr,
    uint8_t* __restrict__ smark, int64_t* __restrict__ slot, const BatchStatus* __restrict__ st) {
  // The new entries whose values fall inside the item's old entries, staged in shared memory,
  // so that each old entry counts the new ones below it there instead of in global memory.
  __shared__ int32_t s_run[kLongChunk];
  __shared__ int32_t s_lo, s_n;
  const int64_t n_items = min((int64_t)st->long_items, item_cap);
  for (int64_t q = blockIdx.x; q < n_items; q += gridDim.x) {
    const unsigned long long item = items[q];
    if (item == kNoLongItem) continue;
    const LongPlan P = plan[item >> 32];
    const int32_t k0 = (int32_t)(uint32_t)item * kLongChunk, k1 = min(P.len, k0 + kLongChunk);
    const int32_t suffix = P.a - P.first;
    const int32_t ko1 = min(k1, suffix);  // the item's old entries: [k0, ko1)
    int32_t run_lo = 0, run_n = -1;       // run_n < 0: not staged
    if (k0 < ko1) {
      if (threadIdx.x == 0) {
        // new entries below the item's first old value, and below its last: the ones between
        // are the only ones that tell its old entries apart
        const int32_t v0 = pool[P.s_old + P.first + k0], v1 = pool[P.s_old + P.first + ko1 - 1];
        int32_t lo = 0, hi = P.c;
        while (lo < hi) {
          const int32_t mid = (lo + hi) >> 1;
          if ((int32_t)(uint32_t)dk[P.i0 + mid] < v0) lo = mid + 1;
          else hi = mid;
        }
        int32_t lo2 = lo, hi2 = P.c;
        while (lo2 < hi2) {
          const int32_t mid = (lo2 + hi2) >> 1;
          if ((int32_t)(uint32_t)dk[P.i0 + mid] < v1) lo2 = mid + 1;
          else hi2 = mid;
        }
        s_lo = lo;
        s_n = lo2 - lo;
      }
      __syncthreads();
      run_lo = s_lo;
      run_n = s_n <= kLongChunk ? s_n : -1;
      for (int32_t t = threadIdx.x; t < run_n; t += kThreads) s_run[t] = (int32_t)(uint32_t)dk[P.i0 + run_lo + t];
      __syncthreads();
    }
    for (int32_t k = k0 + (int32_t)threadIdx.x; k < k1; k += kThreads) {
      int32_t val, pos;
      uint8_t mk;
      if (k < suffix) {  // an old entry: shifts by the new entries below it
        val = pool[P.s_old + P.first + k];
        int32_t lo, hi;
        if (run_n >= 0) {
          lo = 0;
          hi = run_n;
          while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (s_run[mid] < val) lo = mid + 1;
            else hi = mid;
          }
          lo += run_lo;
        } else {
          lo = 0;
          hi = P.c;
          while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if ((int32_t)(uint32_t)dk[P.i0 + mid] < val) lo = mid + 1;
            else hi = mid;
          }
        }
        pos = k + lo;
        mk = 0;
      } else {  // a new entry: lands after the old entries below it
        const int32_t j = k - suffix;
        val = (int32_t)(uint32_t)dk[P.i0 + j];
        pos = j + (int32_t)(lower_bound(pool, P.s_old, P.s_old + P.a, val) - P.s_old) - P.first;
        slot[P.i0 + j] = P.s_new + P.first + pos;
        mk = 1;
      }
      scr[P.soff + pos] = val;
      smark[P.soff + pos] = mk;
    }
    __syncthreads();  // the next item restages s_run
  }
}

__global__ void __launch_bounds__(kThreads) k_long_write(
    const LongPlan* __restrict__ plan, const unsigned long long* __restrict__ items, const int64_t item_cap,
    const int32_t* __restrict__ scr, const uint8_t* __restrict__ smark, int32_t* __restrict__ pool,
    uint8_t* __restrict__ mark, const BatchStatus* __restrict__ st) {
  const int64_t n_items = min((int64_t)st->long_items, item_cap);
  for (int64_t q = blockIdx.x; q < n_items; q += gridDim.x) {
    const unsigned long long item = items[q];
    if (item == kNoLongItem) continue;
    const LongPlan P = plan[item >> 32];
    const int32_t k0 = (int32_t)(uint32_t)item * kLongChunk, k1 = min(P.len, k0 + kLongChunk);
    for (int32_t k = k0 + (int32_t)threadIdx.x; k < k1; k += kThreads) {
      const int64_t dest = P.s_new + P.first + k;
      pool[dest] = scr[P.soff + k];
      if (mark) mark[dest] = smark[P.soff + k];
    }
  }
}

// Deletions from long lists (more than kLongList entries), in four launches over all of the
// batch's long lists at once, through the insertion's scratch buffer:
//   k_cmp_plan    one thread per vertex of the deletions: claims the list (the epoch) and gives it
//                 work items of kLongChunk entries and a range of the scratch;
//   k_cmp_stage   one CTA per item: the chunk's kept entries, compacted within the chunk, into
//                 scratch, and their count; the chunk's marks cleared;
//   k_cmp_prefix  one thread per list: its chunks' output offsets (a prefix of the counts) and
//                 its new length;
//   k_cmp_write   one CTA per item: the chunk's kept entries from scratch to their place.
// The scratch keeps sources and targets apart, so chunks of one list proceed on many CTAs.
struct CmpPlan {
  int64_t s;       // list start
  int64_t soff;    // the list's range in the scratch buffer (chunks j0 on)
  int64_t ib;      // its first work item
  int32_t v;
  int32_t a;       // entries before the deletions
  int32_t nch;     // work items: chunks j0 .. j0 + nch - 1
  int32_t j0;      // the chunk of the first marked slot; the chunks below it stay in place
};

__global__ void __launch_bounds__(kThreads) k_cmp_plan(
    const int32_t* __restrict__ vlist, const int64_t nv_list, const int stride,
    const unsigned long long* __restrict__ nv_dev, const int64_t* __restrict__ start,
    const int32_t* __restrict__ used, unsigned* __restrict__ claim, const unsigned* __restrict__ epoch_dev,
    int32_t* __restrict__ first_del, CmpPlan* __restrict__ plan, unsigned long long* __restrict__ items,
    const int64_t item_cap, const int64_t scr_cap, BatchStatus* __restrict__ st) {
  const unsigned epoch = *epoch_dev;
  const int64_t cnt = nv_dev ? (int64_t)(*nv_dev) * stride : nv_list;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = vlist[k];
    const int32_t a = used[v];
    if (a <= kLongList) continue;  // k_compact_marked's
    if (atomicMax(&claim[v], epoch) >= epoch) continue;  // claimed by another entry of v
    CmpPlan P;
    P.v = v;
    P.a = a;
    P.s = start[v];
    const int32_t f = min(first_del[v], a);
    first_del[v] = kNoDel;
    P.j0 = f / kLongChunk;
    P.nch = f < a ? (a + kLongChunk - 1) / kLongChunk - P.j0 : 0;
    const int32_t span = a - P.j0 * kLongChunk;  // entries from chunk j0 on
    const unsigned long long so = atomicAdd(&st->cmp_scr, (unsigned long long)span);
    const unsigned long long ib = atomicAdd(&st->cmp_items, (unsigned long long)P.nch);
    const unsigned long long r = atomicAdd(&st->n_cmp, 1ull);
    if ((int64_t)(so + span) > scr_cap || (int64_t)(ib + P.nch) > item_cap) {
      atomicOr(&st->err, kErrScratch);  // unreachable while the scratch follows the pool's size
      for (int32_t j = 0; j < P.nch && (int64_t)(ib + j) < item_cap; ++j) items[ib + j] = kNoLongItem;
      P.nch = 0;
    } else {
      for (int32_t j = 0; j < P.nch; ++j) items[ib + j] = (r << 32) | (unsigned)(P.j0 + j);
    }
    P.soff = (int64_t)so;
    P.ib = (int64_t)ib;
    plan[r] = P;
  }
}

// Each thread holds kCmpPer consecutive entries of the chunk (256 threads x 16 = kLongChunk).
constexpr int kCmpPer = kLongChunk / kThreads;
static_assert(kCmpPer % 4 == 0, "a thread's run of entries is whole 16-byte units");

__global__ void __launch_bounds__(kThreads) k_cmp_stage(
    const CmpPlan* __restrict__ plan, const unsigned long long* __restrict__ items, const int64_t item_cap,
    const int32_t* __restrict__ pool, uint8_t* __restrict__ mark, int32_t* __restrict__ scr,
    int2* __restrict__ chunk, const BatchStatus* __restrict__ st) {
  __shared__ int32_t sh_wsum[kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t n_items = min((int64_t)st->cmp_items, item_cap);
  for (int64_t q = blockIdx.x; q < n_items; q += gridDim.x) {
    const unsigned long long item = items[q];
    if (item == kNoLongItem) continue;
    const CmpPlan P = plan[item >> 32];
    const int32_t j = (int32_t)(uint32_t)item;
    const int32_t c0 = j * kLongChunk;
    const int32_t r0 = (j - P.j0) * kLongChunk;  // the chunk's place in the list's scratch range
    const int32_t i0 = c0 + (int32_t)threadIdx.x * kCmpPer;
    int32_t val[kCmpPer];
    unsigned keepm = 0;
    int32_t kept = 0;
    if (i0 + kCmpPer <= P.a) {
      // a full run of kCmpPer entries: 16-byte loads of the entries (list starts are multiples of
      // 4 entries and i0 of kCmpPer) and 4-byte loads of their marks, all independent
      const int4* e4 = reinterpret_cast<const int4*>(pool + P.s + i0);
      uint32_t* m4 = reinterpret_cast<uint32_t*>(mark + P.s + i0);
#pragma unroll
      for (int u = 0; u < kCmpPer / 4; ++u) {
        const int4 v = e4[u];
        const uint32_t m = m4[u];
        val[4 * u] = v.x;
        val[4 * u + 1] = v.y;
        val[4 * u + 2] = v.z;
        val[4 * u + 3] = v.w;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const bool keep = ((m >> (8 * b)) & 0xffu) == 0;
          keepm |= (unsigned)keep << (4 * u + b);
          kept += keep;
        }
        if (m) m4[u] = 0u;  // the deleted slots' marks are cleared (kept slots' are zero)
      }
    } else {
#pragma unroll
      for (int t = 0; t < kCmpPer; ++t) {
        const int32_t i = i0 + t;
        bool keep = false;
        val[t] = 0;
        if (i < P.a) {
          keep = mark[P.s + i] == 0;
          if (keep) val[t] = pool[P.s + i];
          else mark[P.s + i] = 0;
        }
        keepm |= (unsigned)keep << t;
        kept += keep;
      }
    }
    int32_t incl = kept;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) sh_wsum[wid] = incl;
    __syncthreads();
    int32_t before = 0, total = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      const int32_t x = sh_wsum[w];
      if (w < wid) before += x;
      total += x;
    }
    int32_t at = before + incl - kept;
#pragma unroll
    for (int t = 0; t < kCmpPer; ++t)
      if (keepm >> t & 1u) scr[P.soff + r0 + at++] = val[t];
    if (threadIdx.x == 0) chunk[P.ib + (j - P.j0)] = make_int2(0, total);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads) k_cmp_prefix(const CmpPlan* __restrict__ plan, int2* __restrict__ chunk,
                                                         int32_t* __restrict__ used, BatchStatus* __restrict__ st) {
  const int64_t n = (int64_t)st->n_cmp;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const CmpPlan P = plan[r];
    if (P.nch == 0) continue;
    int32_t off = P.j0 * kLongChunk;  // the chunks below j0 keep their entries in place
    for (int32_t j = 0; j < P.nch; ++j) {
      const int32_t c = chunk[P.ib + j].y;
      chunk[P.ib + j].x = off;
      off += c;
    }
    used[P.v] = off;
    atomicAdd(&st->dir_removed, (unsigned long long)(P.a - off));
  }
}

__global__ void __launch_bounds__(kThreads) k_cmp_write(
    const CmpPlan* __restrict__ plan, const unsigned long long* __restrict__ items, const int64_t item_cap,
    const int32_t* __restrict__ scr, const int2* __restrict__ chunk, int32_t* __restrict__ pool,
    const BatchStatus* __restrict__ st) {
  const int64_t n_items = min((int64_t)st->cmp_items, item_cap);
  for (int64_t q = blockIdx.x; q < n_items; q += gridDim.x) {
    const unsigned long long item = items[q];
    if (item == kNoLongItem) continue;
    const CmpPlan P = plan[item >> 32];
    const int32_t j = (int32_t)(uint32_t)item - P.j0;
    const int2 oc = chunk[P.ib + j];
    for (int32_t t = threadIdx.x; t < oc.y; t += kThreads) pool[P.s + oc.x + t] = scr[P.soff + j * kLongChunk + t];
  }
}

// ---- the triangle delta of changed edges -----------------------------------------------------

enum { kPredMark = 0, kPredBatch = 1 };

struct BatchLists {
  const int32_t* src;    // sorted directed entries (cuStinger path)
  const int32_t* dst;
  const int32_t* off;    // batch CSR over src, int32[nv+1]
  const int32_t* dup;
};

struct DeltaArgs {
  SlackView g;
  const uint8_t* mark;
  // entries: either int2/int4 canonical lists (mark predicate) or the batch arrays
  const int2* ilist;
  const int4* dlist;
  const unsigned long long* count_dev;  // number of entries (device), or NULL with count_host
  int64_t count_host;
  BatchLists bl;
  int sign;          // +1 insertions, -1 deletions
  uint32_t weight;   // per-vertex increment per counted triangle
  int search_ratio_x16;
  int only_present;  // skip entries whose edge is absent (cuStinger deletion count)
  int use_table;     // per-cell strategy table: 0 = search, 1 = merge
  int cell_filter;   // -1 all, -2 none, c >= 0 only edges of cell c (timing mode)
  // split queue: (entry << 24 | chunk) items of long intersections (NULL = no splitting)
  unsigned long long* split_items;
  unsigned long long* split_cnt;  // zero before the first pass
  int split_min;     // intersections whose shorter list is longer than this are split ...
  int chunk;         // ... into items of this many entries of the shorter list
  int shard;         // this rank counts the entries e with e % nshards == shard
  int nshards;
  unsigned long long* bytes_out;  // algorithmic bytes of the intersections run (NULL = not kept)
  // persistent kernel (k_delta_fused): its warps take split items while other warps still run
  // the entry pass. An item slot is published by writing the launch's epoch (*item_epoch, bumped
  // before each launch) into item_tag[slot]; entry_done counts the warps done with the entry
  // pass (zero at launch). A wait for an item that runs out reports kErrTimeout in err; bar_extra
  // is added to the warps the item pass waits for (0; a test sets 1 to make the wait run out);
  // spin_ns bounds each wait.
  unsigned* entry_done;
  unsigned* item_tag;
  const unsigned* item_epoch;
  unsigned* err;
  unsigned bar_extra;
  unsigned long long spin_ns;
  // hub-centred counting (k_delta_hub): changed edges whose longer endpoint holds at least
  // hub_min of the phase's changed edges are counted at that endpoint (0 = never); hubbed[e] = 1
  // marks them for the per-edge kernel to skip (NULL = no hub groups)
  int hub_min;
  const uint8_t* hubbed;
  // dynamic work queues of k_delta_fused's two passes (zero at launch; NULL = warp-strided)
  unsigned long long* e_next;
  unsigned long long* i_next;
  int stage_ok;      // the launch has kStageSmem of dynamic shared memory: staged cells may stage
  uint8_t table[256];
};

__device__ __forceinline__ int cell_of(int a, int b) {
  const int ca = min(31 - __clz(max(a, 1)), 15), cb = min(31 - __clz(max(b, 1)), 15);
  return ca * 16 + cb;
}

template <int PRED>
__device__ __forceinline__ bool changed(const DeltaArgs& A, int32_t owner, int64_t slot_abs, int32_t w) {
  if (PRED == kPredMark) return A.mark[slot_abs] != 0;
  const int32_t lo = A.bl.off[owner], hi = A.bl.off[owner + 1];
  int32_t l = lo, h = hi;
  while (l < h) {
    const int32_t mid = (l + h) >> 1;
    if (A.bl.dst[mid] < w) l = mid + 1;
    else h = mid;
  }
  return l < hi && A.bl.dst[l] == w && A.bl.dup[l] == 0;
}

// Entry e of the changed-edge list: its endpoints and whether it adds to the total (the
// cuStinger-style batch holds both directions of every edge; the total counts one).
template <int PRED>
__device__ __forceinline__ bool delta_entry(const DeltaArgs& A, int64_t e, int32_t& x, int32_t& y, bool& count_total) {
  count_total = true;
  if (PRED == kPredMark) {
    if (A.dlist) {
      const int4 d = A.dlist[e];
      x = d.x;
      y = d.y;
    } else {
      const int2 d = A.ilist[e];
      x = d.x;
      y = d.y;
    }
    return true;
  }
  if (A.bl.dup[e]) return false;
  x = A.bl.src[e];
  y = A.bl.dst[e];
  count_total = x < y;
  return x != y;
}

// Intersection strategies of the delta count (the streaming strategy table's values).
enum : int { kStratSearch = 0, kStratMerge = 1, kStratStage = 2 };
constexpr int kStageEntries = 1024;  // entries of the longer list a warp stages per piece
// Dynamic shared memory of a delta kernel launch that may stage (one buffer per warp); a launch
// without it runs the staged cells as merges.
constexpr size_t kStageSmem = sizeof(int32_t) * kStageEntries * (kThreads / 32);

// The two lists of edge {x, y} as the intersection takes them: A the shorter, B the longer.
struct DeltaPair {
  int32_t oa, ob, la, lb;
  int64_t sa, sb;
  uint64_t key;
  int strat;
  int cell;
};

__device__ __forceinline__ DeltaPair delta_pair(const DeltaArgs& A, int32_t x, int32_t y, int32_t lx, int32_t ly,
                                                int64_t sx, int64_t sy) {
  DeltaPair P;
  const bool xs = lx <= ly;
  P.oa = xs ? x : y;
  P.ob = xs ? y : x;
  P.sa = xs ? sx : sy;
  P.sb = xs ? sy : sx;
  P.la = xs ? lx : ly;
  P.lb = xs ? ly : lx;
  P.key = ekey(x, y);
  P.cell = cell_of(P.la, P.lb);
  const int lg = 32 - __clz(P.lb);
  if (A.use_table) {
    const int t = A.table[P.cell];
    P.strat = t == kStratSearch ? kStratSearch : (t == kStratStage && A.stage_ok) ? kStratStage : kStratMerge;
  } else {
    P.strat = 16LL * P.lb > (long long)A.search_ratio_x16 * P.la * lg ? kStratSearch : kStratMerge;
  }
  return P;
}

// The warp intersects entries [i_begin, i_end) of the shorter list with the longer one and
// returns (in every lane) the triangles kept there; each kept common neighbour w gets its
// per-vertex update here, the endpoints get theirs from the caller.
template <int PRED>
__device__ __forceinline__ uint32_t delta_range(const DeltaArgs& A, const DeltaPair& P, int32_t i_begin,
                                                int32_t i_end, uint32_t* __restrict__ pv) {
  const int lane = threadIdx.x & 31;
  const int32_t* L = A.g.ind;
  uint32_t c = 0;
  auto on_match = [&](int64_t ia, int64_t ib, int32_t w) {
    const bool ca = changed<PRED>(A, P.oa, P.sa + ia, w);
    const bool cb = changed<PRED>(A, P.ob, P.sb + ib, w);
    const bool keep = (!ca || P.key < ekey(P.oa, w)) && (!cb || P.key < ekey(P.ob, w));
    if (keep) {
      ++c;
      atomicAdd(&pv[w], A.weight * (uint32_t)A.sign);
    }
  };
  const int64_t sb = P.sb, eb = P.sb + P.lb;
  if (P.strat == kStratStage) {
    // The part of the longer list that can meet entries [i_begin, i_end) of the shorter one,
    // [lo, hi), is staged into this warp's shared-memory buffer in pieces of kStageEntries
    // (cp.async: every copy of a piece in flight at once); each lane then binary-searches one
    // shorter-list entry in the piece. A piece takes the shorter-list entries up to its last
    // entry (the last piece takes the rest), so each is searched once.
    extern __shared__ __align__(16) int32_t s_stage[];  // kStageSmem bytes (A.stage_ok)
    int32_t* buf = s_stage + (threadIdx.x >> 5) * kStageEntries;
    const int32_t a_first = L[P.sa + i_begin], a_last = L[P.sa + i_end - 1];
    const int32_t lo = warp_lower_bound(L + sb, P.lb, a_first);
    const int32_t hi = warp_lower_bound(L + sb, P.lb, a_last + 1);
    int32_t ia = i_begin;
    for (int32_t cb = lo; cb < hi && ia < i_end; cb += kStageEntries) {
      const int32_t n = min(hi - cb, kStageEntries);
      __syncwarp();  // the previous piece's searches are done with the buffer
      for (int32_t k = lane; k < n; k += 32) cp_async4(buf + k, L + sb + cb + k);
      cp_async_wait_all();
      __syncwarp();
      const int32_t bmax = buf[n - 1];
      const bool last = cb + n >= hi;
      while (ia < i_end) {
        const int32_t i = ia + lane;
        const int32_t w = i < i_end ? L[P.sa + i] : INT32_MAX;
        // the lanes that take part are a prefix (the shorter list ascends with the lane)
        const bool in = i < i_end && (last || w <= bmax);
        const int k = __popc(__ballot_sync(kFull, in));
        if (in) {
          int32_t l = 0, h = n;
          while (l < h) {
            const int32_t mid = (l + h) >> 1;
            if (buf[mid] < w) l = mid + 1;
            else h = mid;
          }
          if (l < n && buf[l] == w) on_match(i, (int64_t)cb + l, w);
        }
        __syncwarp();
        ia += k;
        if (k < 32) break;
      }
    }
  } else if (P.strat == kStratSearch) {
    // The first five search levels come from 32 evenly spaced samples of the longer list, one
    // per lane (a single coalesced load): a lane counts the samples below its key with
    // shuffles, then searches memory only inside that bucket.
    // Each lane searches two entries at once (two independent chains of loads in flight).
    const int64_t step = ((int64_t)P.lb + 31) / 32;
    const int32_t smp = (int64_t)lane * step < P.lb ? L[sb + (int64_t)lane * step] : INT32_MAX;
    const int32_t s31 = __shfl_sync(kFull, smp, 31);
    // [lo, hi): the part of the longer list between the samples around w
    auto bucket = [&](const int32_t w, int64_t& lo, int64_t& hi) {
      int pos = 0;  // samples below w (they ascend with the lane)
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if (__shfl_sync(kFull, smp, pos + st - 1) < w) pos += st;
      if (pos == 31 && s31 < w) pos = 32;
      lo = sb + (pos > 0 ? (int64_t)(pos - 1) * step + 1 : 0);
      hi = sb + (pos < 32 ? min((int64_t)pos * step, (int64_t)P.lb) : (int64_t)P.lb);
    };
    for (int32_t base = i_begin; base < i_end; base += 64) {
      const int32_t i = base + lane, i2 = i + 32;
      const bool in = i < i_end, in2 = i2 < i_end;
      const int32_t w = in ? L[P.sa + i] : INT32_MAX;
      const int32_t w2 = in2 ? L[P.sa + i2] : INT32_MAX;
      int64_t lo, hi, lo2, hi2;
      bucket(w, lo, hi);
      bucket(w2, lo2, hi2);
      if (!in) lo = hi;
      if (!in2) lo2 = hi2;
      while (lo < hi || lo2 < hi2) {  // two lower bounds, one step of each per round
        if (lo < hi) {
          const int64_t mid = lo + ((hi - lo) >> 1);
          if (__ldg(L + mid) < w) lo = mid + 1;
          else hi = mid;
        }
        if (lo2 < hi2) {
          const int64_t mid = lo2 + ((hi2 - lo2) >> 1);
          if (__ldg(L + mid) < w2) lo2 = mid + 1;
          else hi2 = mid;
        }
      }
      if (in && lo < eb && L[lo] == w) on_match(i, lo - sb, w);
      if (in2 && lo2 < eb && L[lo2] == w2) on_match(i2, lo2 - sb, w2);
    }
  } else {
    const int32_t len = i_end - i_begin;
    const int32_t per = (len + 31) / 32;
    const int32_t i0 = i_begin + min(len, lane * per), i1 = min(i_end, i0 + per);
    if (i0 < i1) {
      int64_t p = lower_bound(L, sb, eb, L[P.sa + i0]);
      for (int32_t i = i0; i < i1 && p < eb; ++i) {
        const int32_t w = L[P.sa + i];
        while (p < eb && L[p] < w) ++p;
        if (p < eb && L[p] == w) on_match(i, p - sb, w);
      }
    }
  }
  __syncwarp();
  return warp_sum(c);
}

// Per-CTA flush of the kept-triangle total and the algorithmic bytes: one atomic each per CTA.
__device__ __forceinline__ void delta_flush(unsigned long long tri_acc, unsigned long long bytes_acc,
                                            unsigned long long* __restrict__ tri_out,
                                            unsigned long long* __restrict__ bytes_out) {
  __shared__ unsigned long long s_tri[kThreads / 32], s_bytes[kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    s_tri[wid] = tri_acc;
    s_bytes[wid] = bytes_acc;
  }
  __syncwarp();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0, b = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      t += s_tri[w];
      b += s_bytes[w];
    }
    if (t) atomicAdd(tri_out, t);
    if (b && bytes_out) atomicAdd(bytes_out, b);
  }
}

// Rank that counts the changed edge {x, y} of a sharded count: a hash of the edge's canonical
// key, so every rank assigns each edge alike whatever the order of its own lists.
__device__ __forceinline__ int edge_shard(int32_t x, int32_t y, int nshards) {
  uint64_t z = ekey(x, y) + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return (int)((z ^ (z >> 31)) % (uint64_t)nshards);
}

// The triangle delta of the changed edges, one warp per edge (warp-strided; with shards, only
// this rank's edges). An edge whose shorter list is longer than A.split_min (two hubs) would be one
// warp's serial tail of the whole launch: when A.split_items is set it is queued instead as
// items of A.chunk entries of its shorter list, which the item pass spreads over all warps (a
// full queue leaves the edge to this warp). Lane 0 of each warp accumulates the kept triangles
// and the edge's algorithmic bytes.
template <int PRED>
__device__ __forceinline__ void delta_entries(const DeltaArgs& A, uint32_t* __restrict__ pv, const int64_t gw,
                                              const int64_t nw, unsigned long long& tri_acc,
                                              unsigned long long& bytes_acc) {
  const int lane = threadIdx.x & 31;
  const int64_t cnt = A.count_dev ? (int64_t)(*A.count_dev) : A.count_host;
  const unsigned epoch = A.item_tag ? *A.item_epoch : 0u;
  int64_t next = gw, next_end = 0;
  for (;;) {
    // the next entry: warp-strided, or from runs of kGrab entries taken from the queue
    if (A.e_next) {
      if (next >= next_end) {
        unsigned long long g = 0;
        if (lane == 0) g = atomicAdd(A.e_next, (unsigned long long)kGrab);
        g = __shfl_sync(kFull, g, 0);
        if ((int64_t)g >= cnt) break;
        next = (int64_t)g;
        next_end = min(cnt, next + kGrab);
      }
    } else if (next >= cnt) {
      break;
    }
    const int64_t e = next;
    next += A.e_next ? 1 : nw;
    if (A.hubbed && A.hubbed[e]) continue;  // counted at its hub (k_delta_hub)
    int32_t x, y;
    bool count_total;
    if (!delta_entry<PRED>(A, e, x, y, count_total)) continue;
    if (A.nshards > 1 && edge_shard(x, y, A.nshards) != A.shard) continue;
    const int32_t lx = A.g.len(x), ly = A.g.len(y);
    if (lx < 2 || ly < 2) continue;
    const int64_t sx = A.g.start(x), sy = A.g.start(y);
    if (PRED == kPredBatch && A.only_present) {
      // the edge must exist for its triangles to be destroyed
      bool pres = false;
      if (lane == 0) {
        const int64_t p = lower_bound(A.g.ind, sx, sx + lx, y);
        pres = p < sx + lx && A.g.ind[p] == y;
      }
      __syncwarp();
      if (!__shfl_sync(kFull, pres, 0)) continue;
    }
    const DeltaPair P = delta_pair(A, x, y, lx, ly, sx, sy);
    if (A.cell_filter == -2 || (A.cell_filter >= 0 && P.cell != A.cell_filter)) continue;
    if (lane == 0 && count_total) bytes_acc += 4ull * (unsigned long long)(lx + ly) + 8ull;
    if (A.split_items && P.la > A.split_min) {
      const int nch = (P.la + A.chunk - 1) / A.chunk;
      unsigned long long at = 0;
      if (lane == 0) at = atomicAdd(A.split_cnt, (unsigned long long)nch);
      at = __shfl_sync(kFull, at, 0);
      const bool fits = at + (unsigned long long)nch <= (unsigned long long)kDeltaItems;
      for (int j = lane; j < nch; j += 32)
        if (at + j < (unsigned long long)kDeltaItems) {
          A.split_items[at + j] = fits ? ((unsigned long long)e << 24) | (unsigned long long)j : kNoItem;
          if (A.item_tag) st_release(A.item_tag + at + j, epoch);  // the slot is ready
        }
      if (fits) continue;
    }
    const uint32_t c = delta_range<PRED>(A, P, 0, P.la, pv);
    if (lane == 0 && c) {
      atomicAdd(&pv[x], c * A.weight * (uint32_t)A.sign);
      atomicAdd(&pv[y], c * A.weight * (uint32_t)A.sign);
      if (count_total) tri_acc += c;
    }
  }
}

// One queued chunk of a split intersection, run by the warp. The item's edge passed every check
// of the entry pass already; its endpoints' per-vertex updates and the total add up per chunk.
template <int PRED>
__device__ __forceinline__ void delta_item_run(const DeltaArgs& A, uint32_t* __restrict__ pv,
                                               const unsigned long long item, const int64_t cnt,
                                               unsigned long long& tri_acc) {
  const int lane = threadIdx.x & 31;
  if (item == kNoItem) return;
  const int64_t e = (int64_t)(item >> 24);
  const int32_t k = (int32_t)(item & 0xffffffu);
  if (e >= cnt) return;  // only an item of an abandoned pass could hold one
  int32_t x, y;
  bool count_total;
  if (!delta_entry<PRED>(A, e, x, y, count_total)) return;
  const int32_t lx = A.g.len(x), ly = A.g.len(y);
  const int64_t sx = A.g.start(x), sy = A.g.start(y);
  const DeltaPair P = delta_pair(A, x, y, lx, ly, sx, sy);
  const int32_t i0 = k * A.chunk;
  if (i0 >= P.la) return;
  const uint32_t c = delta_range<PRED>(A, P, i0, min(P.la, i0 + A.chunk), pv);
  if (lane == 0 && c) {
    atomicAdd(&pv[x], c * A.weight * (uint32_t)A.sign);
    atomicAdd(&pv[y], c * A.weight * (uint32_t)A.sign);
    if (count_total) tri_acc += c;
  }
}

// The queued chunks of the split intersections after the entry pass has finished (the second
// launch of the cuStinger-style count), one warp per item: warp-strided, or one at a time from
// the queue.
template <int PRED>
__device__ __forceinline__ void delta_items(const DeltaArgs& A, uint32_t* __restrict__ pv, const int64_t gw,
                                            const int64_t nw, unsigned long long& tri_acc) {
  const int lane = threadIdx.x & 31;
  const int64_t n_items = (int64_t)min(*A.split_cnt, (unsigned long long)kDeltaItems);
  const int64_t cnt = A.count_dev ? (int64_t)(*A.count_dev) : A.count_host;
  for (int64_t q0 = gw;;) {
    int64_t q = q0;
    if (A.i_next) {
      unsigned long long g = 0;
      if (lane == 0) g = atomicAdd(A.i_next, 1ull);
      q = (int64_t)__shfl_sync(kFull, g, 0);
    } else {
      q0 += nw;
    }
    if (q >= n_items) break;
    delta_item_run<PRED>(A, pv, A.split_items[q], cnt, tri_acc);
  }
}

// Wait (lane 0 of a warp) until queue slot q holds a published item of this launch: 1 when it
// does, 0 when no item will come to slot q (every warp has finished the entry pass and q lies
// beyond the items they queued, or q beyond the queue's capacity), -1 when the wait ran out
// (spin_ns of device time, at most kSpinMaxIters polls; kErrTimeout is set). A producer publishes
// each slot before it counts itself done, so once every warp is done a reserved slot is ready.
__device__ __forceinline__ int wait_item(const DeltaArgs& A, const unsigned long long q, const unsigned epoch,
                                         const unsigned total) {
  if (q >= (unsigned long long)kDeltaItems) return 0;
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (unsigned it = 0;; ++it) {
    if (ld_acquire(A.item_tag + q) == epoch) return 1;
    if (ld_acquire(A.entry_done) >= total && q >= ld_acquire64(A.split_cnt)) return 0;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (it >= kSpinMaxIters || t - t0 > A.spin_ns) {
      atomicOr(A.err, kErrTimeout);
      return -1;
    }
    __nanosleep(64);
  }
}

// The item pass of the persistent kernel: it starts as soon as the warp's own entry pass ends,
// while other warps may still queue items. Slots are taken in order from the queue head; a slot
// is read once its tag carries this launch's epoch (items written by other CTAs are read past
// the non-coherent L1 after the acquire).
template <int PRED>
__device__ __forceinline__ void delta_items_stream(const DeltaArgs& A, uint32_t* __restrict__ pv,
                                                   unsigned long long& tri_acc) {
  const int lane = threadIdx.x & 31;
  const unsigned epoch = *A.item_epoch;
  const unsigned total = (unsigned)(((int64_t)gridDim.x * blockDim.x) >> 5) + A.bar_extra;
  const int64_t cnt = (int64_t)__ldcg(A.count_dev);
  for (;;) {
    unsigned long long q = 0;
    int state = 0;
    if (lane == 0) {
      q = atomicAdd(A.i_next, 1ull);
      state = wait_item(A, q, epoch, total);
    }
    __syncwarp();
    state = __shfl_sync(kFull, state, 0);
    q = __shfl_sync(kFull, q, 0);
    if (state != 1) break;
    delta_item_run<PRED>(A, pv, __ldcg(A.split_items + q), cnt, tri_acc);
  }
}

// Two launches: the entry pass, then the item pass (the cuStinger-style count, tc_count_batch).
template <int PRED>
__global__ void __launch_bounds__(kThreads, 6) k_delta(const DeltaArgs A, uint32_t* __restrict__ pv,
                                                    unsigned long long* __restrict__ tri_out) {
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long tri_acc = 0, bytes_acc = 0;
  delta_entries<PRED>(A, pv, gw, nw, tri_acc, bytes_acc);
  delta_flush(tri_acc, bytes_acc, tri_out, A.bytes_out);
}

template <int PRED>
__global__ void __launch_bounds__(kThreads, 6) k_delta_split(const DeltaArgs A, uint32_t* __restrict__ pv,
                                                          unsigned long long* __restrict__ tri_out) {
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long tri_acc = 0;
  delta_items<PRED>(A, pv, gw, nw, tri_acc);
  delta_flush(tri_acc, 0ull, tri_out, nullptr);
}

// One persistent launch (a resident grid, at most the occupancy limit of CTAs per SM): every warp
// runs its share of the entry pass, queueing the chunks of split intersections, counts itself
// done, and then takes queued chunks until none is left: no grid-wide barrier, so warps whose
// entry work ends early start on the chunks while others still queue them. The batch size is
// read from device memory, so one captured launch serves every batch of a bin. The launch's
// epoch (bumped before it) marks the slots published in this launch. A wait that runs out (the
// grid was not resident, or a test forces it) sets kErrTimeout and the warp leaves the item
// pass: the batch's count is then incomplete and the host reports TC_ERR_TIMEOUT.
template <int PRED>
#ifndef TC_DELTA_MIN_BLOCKS
#define TC_DELTA_MIN_BLOCKS 6
#endif
__global__ void __launch_bounds__(kThreads, TC_DELTA_MIN_BLOCKS) k_delta_fused(const DeltaArgs A, uint32_t* __restrict__ pv,
                                                          unsigned long long* __restrict__ tri_out) {
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long tri_acc = 0, bytes_acc = 0;
  delta_entries<PRED>(A, pv, gw, nw, tri_acc, bytes_acc);
  // this warp's items are published: count it done (its lanes' releases before lane 0's add)
  __threadfence();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    __threadfence();
    atomicAdd(A.entry_done, 1u);
  }
  delta_items_stream<PRED>(A, pv, tri_acc);
  delta_flush(tri_acc, bytes_acc, tri_out, A.bytes_out);
}

// ---- hub-centred delta count ------------------------------------------------------------------
//
// The changed edges of a batch phase concentrate on few endpoints (R-MAT insertions draw both
// endpoints by degree). An edge {h, s} whose longer-list endpoint h (ties to the smaller id) holds
// at least hub_min of the phase's changed edges is counted at h: a CTA hashes N(h) into shared
// memory, each key with bit 31 set when the edge (h, key) is itself changed (the mark array), and
// its warps stream the partner lists N(s) through the table with coalesced loads, in units of
// kHubUnit entries that the warps take one at a time (a long partner list, another hub's, is
// many units, so no warp holds the others up). Per partner entry that is one shared-memory probe,
// where the per-edge kernel binary-searches it into the longer list. A hub longer than one table
// (kHubPass entries) is hashed in value-range passes: pass pk holds the entries of N(h) in
// [vlo, vhi), and a unit is walked only over its entries in that range (its first and last
// entries tell whether it meets the range; a warp-cooperative sampled search finds where it
// enters), so every partner entry is probed once over the passes. A hub's work is cut into items
// (pass, chunk of its units), each one CTA's table build plus walks, sized so the build is a small
// part of the item; the items of all hubs share one queue, so no hub is a serial tail.
// The keep rule is the per-edge kernel's: a common neighbour w is kept unless (h, w) or (s, w) is
// a changed edge with a smaller key, so every triangle is still attributed to exactly one changed
// edge whichever kernel counts it. Grouping takes three passes over the changed edges: count the
// edges, units and partner entries per longer endpoint, where a vertex becomes a hub when its
// edge count reaches hub_min; give each hub a range of unit slots and its items; place the units
// and flag the edges hubbed. A hub whose units or items do not fit is left to the per-edge kernel.

#ifndef TC_HUB_THREADS
#define TC_HUB_THREADS 512
#endif
constexpr int kHubThreads = TC_HUB_THREADS;
constexpr int kHubCtasPerSm = 1536 / kHubThreads;
constexpr int kHubBucketsMax = 2048 * kHubThreads / 256;  // 64 KB of int32 keys for 512 threads
#ifndef TC_HUB_UNIT
#define TC_HUB_UNIT 512
#endif
// Partner entries per unit of work of a warp. Smaller units shorten the wait at the end of an
// item for the warp with the last unit; on the streaming workload 512 entries measured 5 % less
// time than 1024 over the whole run (prefetching the next 128 entries changed nothing).
constexpr int kHubUnit = TC_HUB_UNIT;
constexpr int kHubPass = 2 * kHubBucketsMax;  // entries of N(h) per pass (load <= 0.5)
constexpr int32_t kHubMarkBit = INT32_MIN;    // bit 31 of a stored key: the edge (h, key) is changed
constexpr int64_t kHubSearchCost = 64;        // an item's estimate of one range search, in probes
#ifndef TC_HUB_ITEM_LOG2
#define TC_HUB_ITEM_LOG2 17
#endif
constexpr int64_t kHubItemMin = 1ll << TC_HUB_ITEM_LOG2;  // probes of work per item at least ...
constexpr int64_t kHubBuildShare = 16;        // ... and at least this many times its table build
constexpr int64_t kHubItemsPerUpdate = 4;     // item queue capacity per batch update
constexpr int64_t kHubUnitsPerUpdate = kHubUnit >= 1024 ? 4 : 4 * 1024 / kHubUnit;  // unit slots per update

struct HubWs {
  int32_t* cnt;      // [n] changed edges per longer endpoint in this phase (zero between phases)
  int32_t* uni;      // [n] their partner units (zero between phases)
  long long* sum;    // [n] sum of their partner list lengths (zero between phases)
  int32_t* of;       // [n] hub id + 1 of a vertex (zero between phases)
  int32_t* list;     // [cap] hub vertices
  int32_t* off;      // [cap] first slot of a hub's units in `units`
  int32_t* len;      // [cap] number of units of the hub
  int32_t* chunks;   // [cap] unit chunks of the hub (items per pass)
  int32_t* fill;     // [cap]
  int2* units;       // [unit_cap] (partner s, unit r: entries [r kHubUnit, (r + 1) kHubUnit) of N(s))
  int64_t unit_cap;
  uint8_t* hubbed;   // [cap] 1 = counted at its hub
  unsigned long long* items;  // [item_cap] (hub id << 32 | item index within the hub)
  int64_t item_cap;
  unsigned long long* n_hubs;
  unsigned long long* total;
  unsigned long long* n_items;
  unsigned long long* q;
};

// Changed edge e as the hub count sees it: false unless this rank counts it and both lists have
// at least two entries (the per-edge kernel's filters); h = the endpoint with the longer list.
__device__ __forceinline__ bool hub_entry(const DeltaArgs& A, int64_t e, int32_t& h, int32_t& s, int32_t& ls) {
  int32_t x, y;
  bool count_total;
  if (!delta_entry<kPredMark>(A, e, x, y, count_total)) return false;
  if (A.nshards > 1 && edge_shard(x, y, A.nshards) != A.shard) return false;
  const int32_t lx = A.g.len(x), ly = A.g.len(y);
  if (lx < 2 || ly < 2) return false;
  const bool x_long = lx > ly || (lx == ly && x < y);
  h = x_long ? x : y;
  s = x_long ? y : x;
  ls = x_long ? ly : lx;
  return true;
}

__global__ void __launch_bounds__(kThreads) k_hub_count(const DeltaArgs A, const HubWs H) {
  const int64_t cnt = (int64_t)*A.count_dev;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
    int32_t h, s, ls;
    if (!hub_entry(A, e, h, s, ls)) continue;
    atomicAdd(reinterpret_cast<unsigned long long*>(&H.sum[h]), (unsigned long long)ls);
    atomicAdd(&H.uni[h], (ls + kHubUnit - 1) / kHubUnit);
    if (atomicAdd(&H.cnt[h], 1) + 1 == A.hub_min) {  // exactly one edge sees the count reach hub_min
      const unsigned long long hid = atomicAdd(H.n_hubs, 1ull);
      H.list[hid] = h;
      H.of[h] = (int32_t)hid + 1;
    }
  }
}

// Passes of a hub of lh entries, and the value range of pass pk: its entries are N(h)[cb, cb_next).
__device__ __forceinline__ int hub_passes(int32_t lh) { return (lh + kHubPass - 1) / kHubPass; }

// Unit slots and items per hub, allocated by atomics; a hub whose units or items do not fit drops
// out (its edges go to the per-edge kernel).
__global__ void __launch_bounds__(kThreads) k_hub_alloc(const DeltaArgs A, const HubWs H) {
  const int64_t nh = (int64_t)*H.n_hubs;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t h = H.list[i];
    const int32_t k = H.uni[h];
    const int32_t lh = A.g.len(h);
    H.len[i] = 0;
    const unsigned long long off = atomicAdd(H.total, (unsigned long long)k);
    if (off + k > (unsigned long long)H.unit_cap) {
      H.of[h] = 0;
      continue;
    }
    const int P = hub_passes(lh);
    // probes of the hub's walks and searches, over the items' target size
    const long long work = H.sum[h] + (long long)(P - 1) * k * kHubSearchCost;
    const long long build = kHubBuildShare * ((long long)lh / P);
    const long long target = build > (long long)kHubItemMin ? build : (long long)kHubItemMin;
    const long long want = (work + target - 1) / target;
    const int C = (int)(want < 1 ? 1 : want > k ? k : want);
    const long long nitems = (long long)P * C;
    const unsigned long long base = atomicAdd(H.n_items, (unsigned long long)nitems);
    if (base + nitems > (unsigned long long)H.item_cap) {
      for (long long j = 0; j < nitems && base + j < (unsigned long long)H.item_cap; ++j) H.items[base + j] = kNoItem;
      H.of[h] = 0;
      continue;
    }
    for (long long j = 0; j < nitems; ++j) H.items[base + j] = ((unsigned long long)i << 32) | (unsigned long long)j;
    H.len[i] = k;
    H.chunks[i] = C;
    H.off[i] = (int32_t)off;
    H.fill[i] = 0;
  }
}

// Place the units of every hub edge in its hub's range and flag the edge; clears the per-vertex
// counts.
__global__ void __launch_bounds__(kThreads) k_hub_place(const DeltaArgs A, const HubWs H) {
  const int64_t cnt = (int64_t)*A.count_dev;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
    uint8_t f = 0;
    int32_t h, s, ls;
    if (hub_entry(A, e, h, s, ls)) {
      const int32_t hid1 = H.of[h];
      if (hid1 > 0) {
        const int32_t u = (ls + kHubUnit - 1) / kHubUnit;
        const int32_t pos = H.off[hid1 - 1] + atomicAdd(&H.fill[hid1 - 1], u);
        for (int32_t r = 0; r < u; ++r) H.units[pos + r] = make_int2(s, r);
        f = 1;
      }
      H.cnt[h] = 0;
      H.uni[h] = 0;
      H.sum[h] = 0;
    }
    H.hubbed[e] = f;
  }
}

__device__ __forceinline__ uint32_t hub_bucket(int32_t w, int bits) {
  return ((uint32_t)w * 0x9E3779B1u) >> (32 - bits);
}

// Insert a key (id, with kHubMarkBit when the edge to it is changed) into 2^bits buckets of 4
// slots (load <= 0.5: a bucket with a free slot is always found).
__device__ __forceinline__ void hub_insert(int32_t* keys, int bits, int32_t id, int32_t key) {
  const uint32_t bmask = (1u << bits) - 1;
  uint32_t b = hub_bucket(id, bits);
  for (uint32_t it = 0; it <= bmask; ++it) {
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if (atomicCAS(&keys[4 * b + t], -1, key) == -1) return;
    b = (b + 1) & bmask;
  }
}

// Is id in the table? If so, `changed` = its stored mark bit (the edge (h, id) is changed).
__device__ __forceinline__ bool hub_find(const int32_t* keys, int bits, int32_t id, bool& changed) {
  const uint32_t bmask = (1u << bits) - 1;
  uint32_t b = hub_bucket(id, bits);
  for (uint32_t it = 0; it <= bmask; ++it) {
    const int4 q = *reinterpret_cast<const int4*>(keys + 4 * b);
    if ((q.x & INT32_MAX) == id) { changed = q.x < 0; return true; }
    if ((q.y & INT32_MAX) == id) { changed = q.y < 0; return true; }
    if ((q.z & INT32_MAX) == id) { changed = q.z < 0; return true; }
    if ((q.w & INT32_MAX) == id) { changed = q.w < 0; return true; }
    if (q.w == -1) return false;  // slots fill in order: a free slot ends the probe
    b = (b + 1) & bmask;
  }
  return false;
}

// Work items of the hubs from one queue: item (hub, j) is pass j / C over unit chunk j % C of the
// hub's C chunks; its warps walk one unit each.
__global__ void __launch_bounds__(kHubThreads, kHubCtasPerSm) k_delta_hub(const DeltaArgs A, const HubWs H,
                                                                          uint32_t* __restrict__ pv,
                                                                          unsigned long long* __restrict__ tri_out) {
  extern __shared__ __align__(16) int32_t hub_keys[];
  __shared__ unsigned long long s_item;
  __shared__ int s_next;
  __shared__ unsigned long long s_red[kHubThreads / 32][2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t n_items = (int64_t)min(*H.n_items, (unsigned long long)H.item_cap);
  const uint32_t inc = A.weight * (uint32_t)A.sign;
  unsigned long long tri_acc = 0, bytes_acc = 0;
  while (true) {
    if (threadIdx.x == 0) {
      const unsigned long long q = atomicAdd(H.q, 1ull);
      s_item = q < (unsigned long long)n_items ? H.items[q] : ~1ull;
      s_next = 0;
    }
    __syncthreads();
    const unsigned long long item = s_item;
    if (item == ~1ull) break;
    if (item == kNoItem) {  // a slot of a hub that did not fit
      __syncthreads();
      continue;
    }
    const int32_t hid = (int32_t)(item >> 32), j = (int32_t)(item & 0xffffffffu);
    const int32_t h = H.list[hid], base = H.off[hid], k = H.len[hid], C = H.chunks[hid];
    const int32_t lh = A.g.len(h);
    const int64_t sh = A.g.start(h);
    const int P = hub_passes(lh);
    const int pk = j / C, ci = j % C;
    const int32_t per = (k + C - 1) / C;
    const int32_t e0 = ci * per, e1 = min(k, e0 + per);
    const int cb = (int)(((int64_t)pk * lh) / P);
    const int cb_next = (int)(((int64_t)(pk + 1) * lh) / P);
    const int clen = cb_next - cb;
    int bits = 4;  // buckets >= clen (load <= 0.25) while they fit, else load <= 0.5
    while ((1 << bits) < clen && (1 << bits) < kHubBucketsMax) ++bits;
    const int S = 4 << bits;
    for (int i = threadIdx.x; i < S; i += kHubThreads) hub_keys[i] = -1;
    __syncthreads();
    for (int i = threadIdx.x; i < clen; i += kHubThreads) {
      const int32_t w = A.g.ind[sh + cb + i];
      hub_insert(hub_keys, bits, w, A.mark[sh + cb + i] ? (w | kHubMarkBit) : w);
    }
    const int32_t vlo = pk == 0 ? INT32_MIN : A.g.ind[sh + cb];
    const int32_t vhi = pk + 1 == P ? INT32_MAX : A.g.ind[sh + cb_next];
    __syncthreads();
    uint32_t hub_c = 0;  // triangles kept at h in this item (lane 0 of each warp)
    while (true) {
      int i = 0;
      if (lane == 0) i = atomicAdd(&s_next, 1);
      i = e0 + __shfl_sync(kFull, i, 0);
      if (i >= e1) break;
      const int2 un = H.units[base + i];
      const int32_t s = un.x;
      const int32_t ls = A.g.len(s);
      const int64_t ss = A.g.start(s);
      const uint64_t key_hs = ekey(h, s);
      if (pk == 0 && un.y == 0 && lane == 0) bytes_acc += 4ull * (unsigned long long)(lh + ls) + 8ull;
      const int32_t c0 = un.y * kHubUnit, c1 = min(ls, c0 + kHubUnit);
      int32_t cur = c0;
      if (P > 1) {  // the unit's part in [vlo, vhi), if any
        const int32_t first = A.g.ind[ss + c0], last = A.g.ind[ss + c1 - 1];
        if (last < vlo || first >= vhi) continue;
        if (first < vlo) cur = c0 + warp_lower_bound(A.g.ind + ss + c0, c1 - c0, vlo);
      }
      uint32_t c = 0;
      // N(s)[cur, c1) up to the first entry >= vhi, 128 entries per step (four loads per lane)
      while (cur < c1) {
        int32_t w[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int32_t q = cur + lane + 32 * t;
          w[t] = q < c1 ? A.g.ind[ss + q] : INT32_MAX;
        }
        int n_in = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const bool in = w[t] < vhi;
          n_in += __popc(__ballot_sync(kFull, in));
          bool ch = false;
          if (in && hub_find(hub_keys, bits, w[t], ch)) {
            const bool cs = A.mark[ss + cur + lane + 32 * t] != 0;
            if ((!ch || key_hs < ekey(h, w[t])) && (!cs || key_hs < ekey(s, w[t]))) {
              ++c;
              atomicAdd(&pv[w[t]], inc);
            }
          }
          __syncwarp();
        }
        cur += n_in;  // the entries below vhi are a prefix of the step (the list ascends)
        if (n_in < 128) break;
      }
      c = warp_sum(c);
      if (lane == 0 && c) {
        atomicAdd(&pv[s], c * inc);
        hub_c += c;
        tri_acc += c;
      }
    }
    // h's per-vertex count: one atomic per item
    if (lane == 0) s_red[wid][0] = hub_c;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0;
      for (int w = 0; w < kHubThreads / 32; ++w) t += s_red[w][0];
      if (t) atomicAdd(&pv[h], (uint32_t)t * inc);
      if (j == 0) H.of[h] = 0;  // zero between phases (k_hub_place, its last reader, is done)
    }
    __syncthreads();
  }
  if (lane == 0) {
    s_red[wid][0] = tri_acc;
    s_red[wid][1] = bytes_acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0, b = 0;
    for (int w = 0; w < kHubThreads / 32; ++w) {
      t += s_red[w][0];
      b += s_red[w][1];
    }
    if (t) atomicAdd(tri_out, t);
    if (b && A.bytes_out) atomicAdd(A.bytes_out, b);
  }
}

// ---- cuStinger-style batch helpers ------------------------------------------------------------

__global__ void k_pack_dir(const int32_t* __restrict__ s, const int32_t* __restrict__ d, const int64_t b,
                           uint64_t* __restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = ((uint64_t)(uint32_t)s[i] << 32) | (uint32_t)d[i];
}

__global__ void k_unpack_dir(const uint64_t* __restrict__ keys, const int64_t b, const int32_t nv, int32_t* __restrict__ s,
                             int32_t* __restrict__ d, int32_t* __restrict__ dup, int32_t* __restrict__ cnt,
                             unsigned* __restrict__ err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const int32_t a = (int32_t)(k >> 32), c = (int32_t)(uint32_t)k;
    s[i] = a;
    d[i] = c;
    const bool bad = a < 0 || a >= nv || c < 0 || c >= nv;
    if (bad) {
      atomicOr(err, kErrRange);
      dup[i] = 1;
      continue;
    }
    dup[i] = (a == c) || (i > 0 && keys[i - 1] == k);
    atomicAdd(&cnt[a], 1);
  }
}

// Entries with dup == 0 that are already in the graph become duplicates; the rest are packed
// as directed insertion keys (sentinel elsewhere).
__global__ void k_flag_present(const SlackView g, const int32_t* __restrict__ s, const int32_t* __restrict__ d,
                               int32_t* __restrict__ dup, const int64_t b, uint64_t* __restrict__ dk) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = kSentinel;
    if (!dup[i]) {
      const int32_t x = s[i], y = d[i];
      const int64_t sx = g.start(x);
      const int32_t lx = g.len(x);
      const int64_t p = lower_bound(g.ind, sx, sx + lx, y);
      if (p < sx + lx && g.ind[p] == y) dup[i] = 1;
      else k = ((uint64_t)(uint32_t)x << 32) | (uint32_t)y;
    }
    dk[i] = k;
  }
}

// Mark the slots of present, non-duplicate entries for deletion; list their source vertices.
__global__ void k_mark_dir_deletions(const SlackView g, const int32_t* __restrict__ s, const int32_t* __restrict__ d,
                                     const int32_t* __restrict__ dup, const int64_t b, uint8_t* __restrict__ mark,
                                     int32_t* __restrict__ first_del, int32_t* __restrict__ vlist,
                                     unsigned long long* __restrict__ nvl) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    if (dup[i]) continue;
    const int32_t x = s[i], y = d[i];
    const int64_t sx = g.start(x);
    const int32_t lx = g.len(x);
    const int64_t p = lower_bound(g.ind, sx, sx + lx, y);
    if (p < sx + lx && g.ind[p] == y) {
      mark[p] = 1;
      atomicMin(&first_del[x], (int32_t)(p - sx));
      vlist[atomicAdd(nvl, 1ull)] = x;
    }
  }
}

__global__ void k_endpoints(const int4* __restrict__ dlist, const BatchStatus* __restrict__ st, int32_t* __restrict__ vlist) {
  const int64_t nd = (int64_t)st->n_del;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += (int64_t)gridDim.x * blockDim.x) {
    vlist[2 * i] = dlist[i].x;
    vlist[2 * i + 1] = dlist[i].y;
  }
}

// The compaction epoch and the delta kernel's item epoch live on the device so that a captured
// launch sequence advances them.
__global__ void k_bump_epoch(unsigned* __restrict__ epoch) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *epoch += 1u;
}

// Canonical keys of a padded batch: entries [b, cap) (b read on the device) become sentinels,
// so a launch sequence sized for cap serves every batch of at most cap updates.
// A device batch into the pipeline's capacity-sized buffers, and its size where the captured
// graph reads it: one launch in place of three copies and a host-to-device copy of the size.
__global__ void k_load_batch(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                             const uint8_t* __restrict__ isdel, const int64_t b, int32_t* __restrict__ wsrc,
                             int32_t* __restrict__ wdst, uint8_t* __restrict__ wdel, int64_t* __restrict__ d_b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
    wsrc[i] = src[i];
    wdst[i] = dst[i];
    wdel[i] = isdel ? isdel[i] : (uint8_t)0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_b = b;
}

__global__ void k_make_keys_cap(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                                const uint8_t* __restrict__ is_del, const int64_t* __restrict__ b_dev,
                                const int64_t cap, const int32_t n, const int L, uint64_t* __restrict__ keys,
                                BatchStatus* __restrict__ st) {
  const uint64_t sent = (1ull << (2 * L + 1)) - 1;
  const int64_t b = min(*b_dev, cap);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = sent;
    if (i < b) {
      const int32_t s = src[i], d = dst[i];
      if (s < 0 || s >= n || d < 0 || d >= n) {
        atomicOr(&st->err, kErrRange);
      } else if (s != d) {
        const uint64_t lo = (uint64_t)min(s, d), hi = (uint64_t)max(s, d);
        k = (lo << (L + 1)) | (hi << 1) | (uint64_t)(is_del[i] ? 0 : 1);
      }
    }
    keys[i] = k;
  }
}

__global__ void k_add_delta(int64_t* __restrict__ delta, const unsigned long long* __restrict__ add,
                            const unsigned long long* __restrict__ sub) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *delta += (int64_t)(add ? *add : 0ull) - (int64_t)(sub ? *sub : 0ull);
}

__global__ void k_to_int32(const int64_t* __restrict__ in, const int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)in[i];
}

}  // namespace

// ---- per-graph streaming workspace -----------------------------------------------------------

struct StreamWs {
  int64_t b_cap = 0;
  int64_t n_cap = 0;
  int32_t* src = nullptr;       // host batches staged here
  int32_t* dst = nullptr;
  uint8_t* isdel = nullptr;
  uint64_t* keys = nullptr;     // [b]
  uint64_t* keys2 = nullptr;    // [b]
  int32_t* head = nullptr;      // [b]
  int4* dlist = nullptr;        // [b]
  int2* ilist = nullptr;        // [b]
  uint64_t* dk = nullptr;       // [2b]
  uint64_t* dk2 = nullptr;      // [2b]
  int32_t* run_start = nullptr; // [2b]
  int32_t* long_runs = nullptr; // [2b] starts of the runs whose list is long
  int32_t* long_cnt = nullptr;  // [2b] their lengths
  LongPlan* long_plan = nullptr;  // [2b]
  CmpPlan* cmp_plan = nullptr;    // [2b] long lists with deletions
  // long-list insertion scratch, sized with the pool (ensure_long_scratch)
  int32_t* long_scr = nullptr;
  uint8_t* long_smark = nullptr;
  unsigned long long* long_items = nullptr;
  int2* long_chunk = nullptr;     // per work item: (output offset, kept entries) of a compacted chunk
  int64_t scr_cap = 0;
  int64_t long_item_cap = 0;
  int64_t* ins_slot = nullptr;  // [2b]
  int32_t* vlist = nullptr;     // [2b]
  unsigned* claim = nullptr;    // [n]
  int32_t* first_del = nullptr; // [n] smallest marked slot of a list in this batch (kNoDel otherwise)
  unsigned* d_epoch = nullptr;  // [1] compaction epoch
  uint64_t version = 0;         // bumped when the batch-sized buffers are reallocated
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  BatchStatus* st = nullptr;
  BatchStatus* st_host = nullptr;  // pinned
  unsigned long long* counter = nullptr;
  int32_t* cnt = nullptr;       // [n+1] per-source counts (cuStinger sort)
  int64_t* scan64 = nullptr;    // [n+1]
  int64_t* tiles = nullptr;
  unsigned long long* split_items = nullptr;  // [kDeltaItems] queued chunks of long intersections
  unsigned* item_tag = nullptr;    // [kDeltaItems] launch epoch that published each item slot
  unsigned* item_epoch = nullptr;  // [1] epoch of the current persistent delta launch
  // hub groups of the delta count (k_delta_hub)
  int32_t* hub_cnt = nullptr;     // [n] zero between phases
  long long* hub_sum = nullptr;   // [n] zero between phases
  int32_t* hub_uni = nullptr;     // [n] zero between phases
  int32_t* hub_of = nullptr;      // [n] zero between phases
  int32_t* hub_list = nullptr;    // [b]
  int32_t* hub_off = nullptr;     // [b]
  int32_t* hub_len = nullptr;     // [b]
  int32_t* hub_fill = nullptr;    // [b]
  int32_t* hub_chunks = nullptr;  // [b]
  int2* hub_units = nullptr;      // [kHubUnitsPerUpdate * b]
  uint8_t* hubbed = nullptr;      // [b]
  unsigned long long* hub_items = nullptr;  // [kHubItemsPerUpdate * b]
  void release();
};

void StreamWs::release() {
  cudaFree(src); cudaFree(dst); cudaFree(isdel); cudaFree(keys); cudaFree(keys2); cudaFree(head);
  cudaFree(dlist); cudaFree(ilist); cudaFree(dk); cudaFree(dk2); cudaFree(run_start); cudaFree(long_runs);
  cudaFree(long_cnt); cudaFree(long_plan); cudaFree(long_scr); cudaFree(long_smark); cudaFree(long_items);
  cudaFree(cmp_plan); cudaFree(long_chunk);
  cudaFree(ins_slot);
  cudaFree(vlist); cudaFree(claim); cudaFree(first_del); cudaFree(d_epoch); cudaFree(cub_tmp); cudaFree(st); cudaFreeHost(st_host); cudaFree(counter);
  cudaFree(cnt); cudaFree(scan64); cudaFree(tiles); cudaFree(split_items); cudaFree(item_tag); cudaFree(item_epoch);
  cudaFree(hub_cnt); cudaFree(hub_sum); cudaFree(hub_uni); cudaFree(hub_of); cudaFree(hub_list); cudaFree(hub_off);
  cudaFree(hub_len); cudaFree(hub_fill); cudaFree(hub_chunks); cudaFree(hub_units); cudaFree(hubbed);
  cudaFree(hub_items);
  *this = StreamWs();
}

void release_stream_ws(StreamWs* w) {
  if (!w) return;
  w->release();
  delete w;
}

namespace {

// Allocate (or grow) the batch workspace. Each group of arrays is replaced as a whole: a failed
// allocation frees the group and leaves its capacity at 0, so a later call allocates it again and
// no kernel sees a freed or missing array (the graph itself is untouched).
tc_status ensure_stream_ws(tc_graph* g, int64_t b) {
  if (!g->sw) g->sw = new StreamWs();
  StreamWs& w = *g->sw;
  if (!g->mark) {
    uint8_t* mk = nullptr;
    if (::tc::dev_malloc(&mk, (size_t)std::max<int64_t>(g->pool_cap, 1)) != cudaSuccess)
      return fail(TC_ERR_OOM, "edge marks: device allocation failed");
    const cudaError_t e = cudaMemset(mk, 0, (size_t)std::max<int64_t>(g->pool_cap, 1));
    if (e != cudaSuccess) {
      cudaFree(mk);
      return fail(TC_ERR_CUDA, "edge marks: %s", cudaGetErrorString(e));
    }
    g->mark = mk;
  }
  if (w.n_cap < (int64_t)g->n + 1) {
    auto free_pv = [&w]() {
      cudaFree(w.claim); cudaFree(w.first_del); cudaFree(w.cnt); cudaFree(w.scan64); cudaFree(w.tiles);
      cudaFree(w.d_epoch);
      cudaFree(w.hub_cnt); cudaFree(w.hub_sum); cudaFree(w.hub_uni); cudaFree(w.hub_of);
      w.claim = nullptr; w.first_del = nullptr; w.cnt = nullptr; w.scan64 = nullptr; w.tiles = nullptr;
      w.d_epoch = nullptr;
      w.hub_cnt = nullptr; w.hub_sum = nullptr; w.hub_uni = nullptr; w.hub_of = nullptr;
      w.n_cap = 0;
    };
    free_pv();
    ++w.version;
    const size_t n1 = (size_t)g->n + 1;
    if (::tc::dev_malloc(&w.claim, sizeof(unsigned) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.first_del, sizeof(int32_t) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.d_epoch, sizeof(unsigned)) != cudaSuccess ||
        ::tc::dev_malloc(&w.cnt, sizeof(int32_t) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.scan64, sizeof(int64_t) * (n1 + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&w.tiles, sizeof(int64_t) * (size_t)(scan_tiles(g->n + 1) + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&w.hub_cnt, sizeof(int32_t) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.hub_sum, sizeof(long long) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.hub_uni, sizeof(int32_t) * n1) != cudaSuccess ||
        ::tc::dev_malloc(&w.hub_of, sizeof(int32_t) * n1) != cudaSuccess) {
      free_pv();
      return fail(TC_ERR_OOM, "batch workspace (per vertex): device allocation failed");
    }
    TC_CUDA_TRY(cudaMemset(w.claim, 0, sizeof(unsigned) * n1));
    TC_CUDA_TRY(cudaMemset(w.first_del, 0x7f, sizeof(int32_t) * n1));  // kNoDel
    TC_CUDA_TRY(cudaMemset(w.d_epoch, 0, sizeof(unsigned)));
    TC_CUDA_TRY(cudaMemset(w.hub_cnt, 0, sizeof(int32_t) * n1));
    TC_CUDA_TRY(cudaMemset(w.hub_sum, 0, sizeof(long long) * n1));
    TC_CUDA_TRY(cudaMemset(w.hub_uni, 0, sizeof(int32_t) * n1));
    TC_CUDA_TRY(cudaMemset(w.hub_of, 0, sizeof(int32_t) * n1));
    w.n_cap = g->n + 1;
  }
  if (!w.st || !w.st_host || !w.counter || !w.split_items || !w.item_tag || !w.item_epoch) {
    auto free_st = [&w]() {
      cudaFree(w.st); cudaFreeHost(w.st_host); cudaFree(w.counter); cudaFree(w.split_items);
      cudaFree(w.item_tag); cudaFree(w.item_epoch);
      w.st = nullptr; w.st_host = nullptr; w.counter = nullptr; w.split_items = nullptr;
      w.item_tag = nullptr; w.item_epoch = nullptr;
    };
    free_st();
    if (::tc::dev_malloc(&w.st, sizeof(BatchStatus)) != cudaSuccess ||
        cudaMallocHost(&w.st_host, sizeof(BatchStatus)) != cudaSuccess ||
        ::tc::dev_malloc(&w.counter, sizeof(unsigned long long)) != cudaSuccess ||
        ::tc::dev_malloc(&w.split_items, sizeof(unsigned long long) * kDeltaItems) != cudaSuccess ||
        ::tc::dev_malloc(&w.item_tag, sizeof(unsigned) * kDeltaItems) != cudaSuccess ||
        ::tc::dev_malloc(&w.item_epoch, sizeof(unsigned)) != cudaSuccess) {
      free_st();
      return fail(TC_ERR_OOM, "batch status: allocation failed");
    }
    TC_CUDA_TRY(cudaMemset(w.item_tag, 0, sizeof(unsigned) * kDeltaItems));
    TC_CUDA_TRY(cudaMemset(w.item_epoch, 0, sizeof(unsigned)));
    ++w.version;
  }
  if (b <= w.b_cap) return TC_OK;
  const int64_t nb = std::max<int64_t>(b, 1024);
  auto free_batch = [&w]() {
    cudaFree(w.src); cudaFree(w.dst); cudaFree(w.isdel); cudaFree(w.keys); cudaFree(w.keys2); cudaFree(w.head);
    cudaFree(w.dlist); cudaFree(w.ilist); cudaFree(w.dk); cudaFree(w.dk2); cudaFree(w.run_start);
    cudaFree(w.long_runs); cudaFree(w.ins_slot); cudaFree(w.vlist); cudaFree(w.cub_tmp);
    cudaFree(w.long_cnt); cudaFree(w.long_plan); cudaFree(w.cmp_plan);
    w.long_cnt = nullptr; w.long_plan = nullptr; w.cmp_plan = nullptr;
    cudaFree(w.hub_list); cudaFree(w.hub_off); cudaFree(w.hub_len); cudaFree(w.hub_fill); cudaFree(w.hub_chunks);
    cudaFree(w.hub_units); cudaFree(w.hubbed); cudaFree(w.hub_items);
    w.src = nullptr; w.dst = nullptr; w.isdel = nullptr; w.keys = nullptr; w.keys2 = nullptr; w.head = nullptr;
    w.dlist = nullptr; w.ilist = nullptr; w.dk = nullptr; w.dk2 = nullptr; w.run_start = nullptr;
    w.long_runs = nullptr; w.ins_slot = nullptr; w.vlist = nullptr; w.cub_tmp = nullptr;
    w.hub_list = nullptr; w.hub_off = nullptr; w.hub_len = nullptr; w.hub_fill = nullptr; w.hub_chunks = nullptr;
    w.hub_units = nullptr; w.hubbed = nullptr; w.hub_items = nullptr;
    w.b_cap = 0;
    w.cub_bytes = 0;
  };
  free_batch();
  ++w.version;
  size_t t1 = 0, t2 = 0;
  bool ok = ::tc::dev_malloc(&w.src, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.dst, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.isdel, nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.keys, sizeof(uint64_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.keys2, sizeof(uint64_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.head, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.dlist, sizeof(int4) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.ilist, sizeof(int2) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.dk, sizeof(uint64_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.dk2, sizeof(uint64_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.run_start, sizeof(int32_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.long_runs, sizeof(int32_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.long_cnt, sizeof(int32_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.long_plan, sizeof(LongPlan) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.cmp_plan, sizeof(CmpPlan) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.ins_slot, sizeof(int64_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.vlist, sizeof(int32_t) * 2 * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_list, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_off, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_len, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_fill, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_chunks, sizeof(int32_t) * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_units, sizeof(int2) * kHubUnitsPerUpdate * nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hubbed, nb) == cudaSuccess &&
            ::tc::dev_malloc(&w.hub_items, sizeof(unsigned long long) * kHubItemsPerUpdate * nb) == cudaSuccess &&
            cub::DeviceRadixSort::SortKeys(nullptr, t1, w.keys, w.keys2, (int)(2 * nb)) == cudaSuccess &&
            cub::DeviceRadixSort::SortKeys(nullptr, t2, w.dk, w.dk2, (int)(2 * nb)) == cudaSuccess &&
            ::tc::dev_malloc(&w.cub_tmp, std::max(t1, t2)) == cudaSuccess;
  if (!ok) {
    free_batch();
    return fail(TC_ERR_OOM, "batch workspace for %lld updates: device allocation failed", (long long)nb);
  }
  w.cub_bytes = std::max(t1, t2);
  w.b_cap = nb;
  return TC_OK;
}

// Scratch of the long-list insertion: the merged suffixes of one batch's long lists, at most every
// entry of the pool plus the batch's new ones (pool_cap + 2 b), and their work items. Follows the
// pool's capacity; a reallocation bumps the workspace version (captured graphs hold the pointers).
tc_status ensure_long_scratch(tc_graph* g) {
  if (!g->sw) return TC_OK;
  StreamWs& w = *g->sw;
  const int64_t need = g->pool_cap + 2 * w.b_cap;
  if (w.scr_cap >= need && w.long_scr && w.long_smark && w.long_items && w.long_chunk) return TC_OK;
  cudaFree(w.long_scr);
  cudaFree(w.long_smark);
  cudaFree(w.long_items);
  cudaFree(w.long_chunk);
  w.long_scr = nullptr;
  w.long_smark = nullptr;
  w.long_items = nullptr;
  w.long_chunk = nullptr;
  w.scr_cap = 0;
  w.long_item_cap = 0;
  ++w.version;
  const int64_t cap = need + need / 4;
  const int64_t icap = cap / kLongChunk + 2 * w.b_cap + 1;
  if (::tc::dev_malloc(&w.long_scr, sizeof(int32_t) * (size_t)cap) != cudaSuccess ||
      ::tc::dev_malloc(&w.long_smark, (size_t)cap) != cudaSuccess ||
      ::tc::dev_malloc(&w.long_items, sizeof(unsigned long long) * (size_t)icap) != cudaSuccess ||
      ::tc::dev_malloc(&w.long_chunk, sizeof(int2) * (size_t)icap) != cudaSuccess) {
    cudaFree(w.long_scr);
    cudaFree(w.long_smark);
    cudaFree(w.long_items);
    cudaFree(w.long_chunk);
    w.long_scr = nullptr;
    w.long_smark = nullptr;
    w.long_items = nullptr;
    w.long_chunk = nullptr;
    return fail(TC_ERR_OOM, "long-list insertion scratch: device allocation failed");
  }
  w.scr_cap = cap;
  w.long_item_cap = icap;
  return TC_OK;
}

// Make room for `extra` slots past pool_top (grow the pool and the mark array by copying), and
// size the long-list insertion scratch to the pool.
tc_status ensure_pool(tc_graph* g, int64_t extra, cudaStream_t s) {
  const int64_t need = g->pool_top + extra;
  if (need <= g->pool_cap) return ensure_long_scratch(g);
  const int64_t ncap = std::max<int64_t>(need + need / 4, g->pool_cap * 3 / 2);
  int32_t* np = nullptr;
  uint8_t* nm = nullptr;
  if (::tc::dev_malloc(&np, sizeof(int32_t) * (size_t)ncap) != cudaSuccess ||
      ::tc::dev_malloc(&nm, (size_t)ncap) != cudaSuccess) {
    cudaFree(np);
    cudaFree(nm);
    return fail(TC_ERR_OOM, "adjacency pool growth to %lld slots: device allocation failed", (long long)ncap);
  }
  TC_CUDA_TRY(cudaMemcpyAsync(np, g->pool, sizeof(int32_t) * (size_t)g->pool_top, cudaMemcpyDeviceToDevice, s));
  TC_CUDA_TRY(cudaMemsetAsync(nm, 0, (size_t)ncap, s));
  if (g->mark) TC_CUDA_TRY(cudaMemcpyAsync(nm, g->mark, (size_t)g->pool_top, cudaMemcpyDeviceToDevice, s));
  TC_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(g->pool);
  cudaFree(g->mark);
  g->pool = np;
  g->mark = nm;
  g->pool_cap = ncap;
  g->view_version++;
  return ensure_long_scratch(g);
}

int bits_for(int32_t n) {
  int L = 1;
  while (L < 31 && ((int64_t)1 << L) < (int64_t)n) ++L;
  return L;
}

DeltaArgs delta_args(tc_graph* g, const SchedParams& sp) {
  DeltaArgs A;
  memset(&A, 0, sizeof(A));
  A.g = SlackView{g->start, g->used, g->pool};
  A.mark = g->mark;
  A.search_ratio_x16 = sp.search_ratio_x16;
  A.use_table = sp.use_table;
  A.cell_filter = sp.cell_filter;
  A.split_min = kDeltaSplit;
  A.chunk = kDeltaChunk;
  A.shard = sp.shard;
  A.nshards = sp.nshards;
  A.spin_ns = kSpinNs;
  A.hub_min = sp.hub_min;
  memcpy(A.table, sp.table, sizeof(A.table));
  // staging buffers only for launches whose strategy table stages somewhere
  if (A.use_table)
    for (int c = 0; c < 256; ++c) A.stage_ok |= A.table[c] == kStratStage;
  return A;
}

// Dynamic shared memory of a delta-kernel launch with these arguments.
size_t delta_smem(const DeltaArgs& A) { return A.stage_ok ? kStageSmem : 0; }

int delta_grid() { return device_info().sms * 8; }
int long_grid() { return device_info().sms * 8; }

// Deletions from the batch's long lists (k_cmp_plan, k_cmp_stage, k_cmp_prefix, k_cmp_write): the
// vertices vlist[0 .. nv) (nv = nv_dev * stride when nv_dev is set, else nv_list, at most
// nv_cap). The scratch must be sized (ensure_long_scratch).
void long_compact(tc_graph* g, StreamWs& w, const int32_t* vlist, int64_t nv_list, int stride,
                  const unsigned long long* nv_dev, int64_t nv_cap, cudaStream_t s) {
  k_cmp_plan<<<grid_for(nv_cap, kThreads), kThreads, 0, s>>>(vlist, nv_list, stride, nv_dev, g->start, g->used, w.claim,
                                                            w.d_epoch, w.first_del, w.cmp_plan, w.long_items,
                                                            w.long_item_cap, w.scr_cap, w.st);
  k_cmp_stage<<<long_grid(), kThreads, 0, s>>>(w.cmp_plan, w.long_items, w.long_item_cap, g->pool, g->mark, w.long_scr,
                                               w.long_chunk, w.st);
  k_cmp_prefix<<<grid_for(nv_cap, kThreads), kThreads, 0, s>>>(w.cmp_plan, w.long_chunk, g->used, w.st);
  k_cmp_write<<<long_grid(), kThreads, 0, s>>>(w.cmp_plan, w.long_items, w.long_item_cap, w.long_scr, w.long_chunk,
                                               g->pool, w.st);
}

// Insertion into the batch's long lists (k_long_plan, k_long_stage, k_long_write); `nd_cap` bounds
// the long runs (the directed entries' capacity). The scratch must be sized (ensure_pool).
void long_insert(tc_graph* g, StreamWs& w, int64_t nd_cap, uint8_t* mark, cudaStream_t s) {
  k_long_plan<<<grid_for(nd_cap, kThreads), kThreads, 0, s>>>(
      w.dk2, w.long_runs, w.long_cnt, g->start, g->used, g->cap, g->pool, g->pool_cap, w.ins_slot, g->d_pool_top,
      g->slack_q10, w.long_plan, w.long_items, w.long_item_cap, w.scr_cap, w.st);
  k_long_stage<<<long_grid(), kThreads, 0, s>>>(w.dk2, g->pool, w.long_plan, w.long_items, w.long_item_cap, w.long_scr,
                                                w.long_smark, w.ins_slot, w.st);
  k_long_write<<<long_grid(), kThreads, 0, s>>>(w.long_plan, w.long_items, w.long_item_cap, w.long_scr, w.long_smark,
                                                g->pool, mark, w.st);
}

// Grid of the persistent delta kernel: ctas_per_sm CTAs per SM (0 = the occupancy limit), never
// more than can be resident at once (its item pass waits for every warp's entry pass).
tc_status fused_grid(int ctas_per_sm, size_t smem, int* grid) {
  constexpr int kMaxDev = 64;
  static int occ[kMaxDev][2] = {};  // without, with the staging buffers
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  const int k = smem > 0 ? 1 : 0;
  if (occ[dev][k] == 0) {
    int b = 0;
    TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_delta_fused<kPredMark>, kThreads, k ? kStageSmem : 0));
    occ[dev][k] = std::max(1, b);
  }
  const int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, occ[dev][k]) : occ[dev][k];
  *grid = device_info().sms * per_sm;
  return TC_OK;
}

constexpr size_t kHubSmem = sizeof(int32_t) * 4 * kHubBucketsMax;

// Grid of the hub kernel: its occupancy limit of CTAs per SM (64 KB of shared memory each).
tc_status hub_grid(int* grid) {
  constexpr int kMaxDev = 64;
  static int occ[kMaxDev] = {};
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return fail(TC_ERR_INVALID_ARG, "device %d out of range", dev);
  if (occ[dev] == 0) {
    TC_CUDA_TRY(cudaFuncSetAttribute(k_delta_hub, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHubSmem));
    int b = 0;
    TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_delta_hub, kHubThreads, kHubSmem));
    occ[dev] = std::max(1, b);
  }
  *grid = device_info().sms * occ[dev];
  return TC_OK;
}

// Hub groups and their count for one phase of a batch (deletions: phase 0, insertions: 1) on a
// grid of `grid` hub CTAs; `cap` bounds the phase's changed edges. Sets A.hubbed for the
// per-edge kernel that follows (NULL when the hub count is off: hub_min <= 0, or a timing run of
// one degree cell). Launches only (it can run inside a stream capture).
void hub_kernels(DeltaArgs& A, StreamWs& w, int phase, int64_t cap, int grid, uint32_t* pv,
                 unsigned long long* tri_out, cudaStream_t s) {
  A.hubbed = nullptr;
  if (A.hub_min <= 0 || A.cell_filter != -1) return;
  HubWs H;
  H.cnt = w.hub_cnt;
  H.sum = w.hub_sum;
  H.uni = w.hub_uni;
  H.of = w.hub_of;
  H.list = w.hub_list;
  H.off = w.hub_off;
  H.len = w.hub_len;
  H.chunks = w.hub_chunks;
  H.fill = w.hub_fill;
  H.units = w.hub_units;
  H.unit_cap = kHubUnitsPerUpdate * w.b_cap;
  H.hubbed = w.hubbed;
  H.items = w.hub_items;
  H.item_cap = kHubItemsPerUpdate * w.b_cap;
  H.n_hubs = &w.st->n_hubs[phase];
  H.total = &w.st->hub_total[phase];
  H.n_items = &w.st->hub_items[phase];
  H.q = &w.st->hub_q[phase];
  const int gb = grid_for(cap, kThreads);
  k_hub_count<<<gb, kThreads, 0, s>>>(A, H);
  k_hub_alloc<<<gb, kThreads, 0, s>>>(A, H);
  k_hub_place<<<gb, kThreads, 0, s>>>(A, H);
  k_delta_hub<<<grid, kHubThreads, kHubSmem, s>>>(A, H, pv, tri_out);
  A.hubbed = w.hubbed;
}

tc_status launch_hub(DeltaArgs& A, StreamWs& w, int phase, int64_t cap, uint32_t* pv, unsigned long long* tri_out,
                     cudaStream_t s) {
  int grid = 0;
  TC_TRY(hub_grid(&grid));
  hub_kernels(A, w, phase, cap, grid, pv, tri_out, s);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

// The persistent delta kernel of one phase of a batch (deletions: phase 0, insertions: 1) on
// the batch workspace's counters, after the hub groups' count.
tc_status launch_delta_fused(DeltaArgs A, StreamWs& w, int phase, uint32_t* pv, unsigned long long* tri_out,
                             int ctas_per_sm, cudaStream_t s) {
  A.split_items = w.split_items;
  A.split_cnt = &w.st->n_split[phase];
  A.entry_done = &w.st->entry_done[phase];
  A.item_tag = w.item_tag;
  A.item_epoch = w.item_epoch;
  A.err = &w.st->err;
  A.bytes_out = &w.st->delta_bytes;
  A.e_next = &w.st->e_next[phase];
  A.i_next = &w.st->i_next[phase];
  TC_TRY(launch_hub(A, w, phase, w.b_cap, pv, tri_out, s));
  int grid = 0;
  TC_TRY(fused_grid(ctas_per_sm, delta_smem(A), &grid));
  k_bump_epoch<<<1, 32, 0, s>>>(w.item_epoch);  // marks the item slots this launch publishes
  k_delta_fused<kPredMark><<<grid, kThreads, delta_smem(A), s>>>(A, pv, tri_out);
  return TC_OK;
}

}  // namespace
}  // namespace tc

using namespace tc;

extern "C" {

tc_status tc_apply_batch(tc_graph* g, const int32_t* src, const int32_t* dst, const uint8_t* is_delete, int64_t b,
                         int mem, int32_t* per_vertex, int64_t* delta_dev, tc_batch_info* info, const tc_sched* sched,
                         void* stream) {
  tc::TraceRange trace_range("tc_apply_batch");
  if (!g) return fail(TC_ERR_INVALID_ARG, "graph is NULL");
  if (b < 0 || (b > 0 && (!src || !dst)) || (mem != TC_MEM_HOST && mem != TC_MEM_DEVICE))
    return fail(TC_ERR_INVALID_ARG, "invalid batch arguments");
  if (b > (int64_t)INT32_MAX / 2) return fail(TC_ERR_CAPACITY, "batch of %lld pairs exceeds 2^30", (long long)b);
  cudaStream_t s = (cudaStream_t)stream;
  TC_TRY(ensure_stream_ws(g, b));
  StreamWs& w = *g->sw;
  const SchedParams sp = to_params(sched);
  TC_CUDA_TRY(cudaMemsetAsync(w.st, 0, sizeof(BatchStatus), s));
  const int32_t* d_src = src;
  const int32_t* d_dst = dst;
  const uint8_t* d_del = is_delete;
  if (mem == TC_MEM_HOST && b > 0) {
    TC_CUDA_TRY(cudaMemcpyAsync(w.src, src, sizeof(int32_t) * b, cudaMemcpyHostToDevice, s));
    TC_CUDA_TRY(cudaMemcpyAsync(w.dst, dst, sizeof(int32_t) * b, cudaMemcpyHostToDevice, s));
    if (is_delete) TC_CUDA_TRY(cudaMemcpyAsync(w.isdel, is_delete, b, cudaMemcpyHostToDevice, s));
    d_src = w.src;
    d_dst = w.dst;
    d_del = is_delete ? w.isdel : nullptr;
  }
  const int L = bits_for(std::max(g->n, 2));
  const uint64_t sent = (1ull << (2 * L + 1)) - 1;
  SlackView view{g->start, g->used, g->pool};
  const int gb = grid_for(std::max<int64_t>(b, 1), kThreads);
  // 1. canonical keys, sort, unique + classify
  if (b > 0) {
    k_make_keys<<<gb, kThreads, 0, s>>>(d_src, d_dst, d_del, b, g->n, L, w.keys, w.st);
    size_t tb = w.cub_bytes;
    TC_CUDA_TRY(cub::DeviceRadixSort::SortKeys(w.cub_tmp, tb, w.keys, w.keys2, (int)b, 0, 2 * L + 1, s));
    k_run_heads<<<gb, kThreads, 0, s>>>(w.keys2, b, sent, w.head);
    TC_CUDA_TRY(cudaMemsetAsync(w.dk, 0xff, sizeof(uint64_t) * 2 * b, s));
    k_classify<<<gb, kThreads, 0, s>>>(view, w.keys2, b, L, w.head, w.dlist, w.ilist, w.dk, w.st);
    size_t tb2 = w.cub_bytes;
    TC_CUDA_TRY(cub::DeviceRadixSort::SortKeys(w.cub_tmp, tb2, w.dk, w.dk2, (int)(2 * b), 0, 64, s));
    k_dir_runs<<<grid_for(2 * b, kThreads), kThreads, 0, s>>>(w.dk2, 2 * b, g->used, g->cap, g->slack_q10, w.run_start, w.long_runs, w.long_cnt, w.st);
    TC_CUDA_TRY(cudaGetLastError());
  }
  // 2. one synchronisation: sizes and the pool demand
  TC_CUDA_TRY(cudaMemcpyAsync(w.st_host, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaMemcpyAsync(&w.st_host->pool_top, g->d_pool_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaStreamSynchronize(s));
  const BatchStatus h = *w.st_host;
  g->pool_top = (int64_t)h.pool_top;
  if (h.err & kErrRange) return fail(TC_ERR_INVALID_ARG, "batch has vertex ids outside [0, %d)", g->n);
  TC_TRY(ensure_pool(g, (int64_t)h.demand, s));
  uint32_t* pv = reinterpret_cast<uint32_t*>(per_vertex);
  uint32_t* pv_use = pv;
  uint32_t* scratch_pv = nullptr;
  if (!pv_use) {
    // counts only: route per-vertex updates to a scratch array
    if (!g->pv_scratch && ::tc::dev_malloc(&g->pv_scratch, sizeof(uint32_t) * ((size_t)g->n + 1)) != cudaSuccess) {
      g->pv_scratch = nullptr;
      return fail(TC_ERR_OOM, "per-vertex scratch: device allocation failed");
    }
    scratch_pv = reinterpret_cast<uint32_t*>(g->pv_scratch);
    pv_use = scratch_pv;
  }
  view = SlackView{g->start, g->used, g->pool};
  // 3. deletions: mark, count on the pre-deletion graph, compact
  if (h.n_del > 0) {
    const int gd = grid_for((int64_t)h.n_del, kThreads);
    k_mark_deletions<<<gd, kThreads, 0, s>>>(w.dlist, w.st, g->start, g->mark, w.first_del);
    DeltaArgs A = delta_args(g, sp);
    A.dlist = w.dlist;
    A.count_dev = &w.st->n_del;
    A.sign = -1;
    A.weight = 2;
    TC_TRY(launch_delta_fused(A, w, 0, pv_use, &w.st->tri_removed, 0, s));
    k_endpoints<<<gd, kThreads, 0, s>>>(w.dlist, w.st, w.vlist);
    k_bump_epoch<<<1, 32, 0, s>>>(w.d_epoch);
    k_compact_marked<<<grid_for(2 * (int64_t)h.n_del * 32, kThreads), kThreads, 0, s>>>(
        w.vlist, 2 * (int64_t)h.n_del, 1, nullptr, g->start, g->used, g->pool, g->mark, w.claim, w.d_epoch,
        w.first_del, w.st);
    long_compact(g, w, w.vlist, 2 * (int64_t)h.n_del, 1, nullptr, 2 * (int64_t)h.n_del, s);
    TC_CUDA_TRY(cudaGetLastError());
  }
  // 4. insertions: merge into the lists, count on the post-insertion graph, clear marks
  if (h.n_ins > 0) {
    k_insert_runs<<<grid_for((int64_t)h.n_runs * 32, kThreads), kThreads, 0, s>>>(
        w.dk2, 2 * b, w.run_start, g->start, g->used, g->cap, g->pool, g->pool_cap, g->mark, w.ins_slot,
        g->d_pool_top, g->slack_q10, w.st);
    long_insert(g, w, 2 * b, g->mark, s);
    DeltaArgs A = delta_args(g, sp);
    A.ilist = w.ilist;
    A.count_dev = &w.st->n_ins;
    A.sign = 1;
    A.weight = 2;
    TC_TRY(launch_delta_fused(A, w, 1, pv_use, &w.st->tri_added, 0, s));
    k_clear_slots<<<grid_for(2 * (int64_t)h.n_ins, kThreads), kThreads, 0, s>>>(w.ins_slot, 2 * (int64_t)h.n_ins,
                                                                                  nullptr, g->mark);
    TC_CUDA_TRY(cudaGetLastError());
  }
  g->m += 2 * ((int64_t)h.n_ins - (int64_t)h.n_del);
  g->pool_top += (int64_t)h.demand;  // host bound until the next read of the device counter
  g->view_version++;
  if (delta_dev) k_add_delta<<<1, 32, 0, s>>>(delta_dev, &w.st->tri_added, &w.st->tri_removed);
  if (info) {
    TC_CUDA_TRY(cudaMemcpyAsync(w.st_host, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaStreamSynchronize(s));
    const BatchStatus& f = *w.st_host;
    if (f.err & (kErrPool | kErrScratch)) return fail(TC_ERR_CAPACITY, "adjacency pool or insertion scratch exhausted");
    if (f.err & kErrTimeout) return fail(TC_ERR_TIMEOUT, "the delta kernel gave up waiting for queued work");
    info->updates = b;
    info->inserted = (int64_t)f.n_ins;
    info->deleted = (int64_t)f.n_del;
    info->ignored = b - (int64_t)f.n_ins - (int64_t)f.n_del;
    info->triangles_added = (int64_t)f.tri_added;
    info->triangles_removed = (int64_t)f.tri_removed;
    info->status = TC_OK;
  }
  return TC_OK;
}

tc_status tc_batch_sort(int32_t nv, int32_t* d_src, int32_t* d_dst, int64_t b, int32_t* d_offsets, int32_t* d_dup,
                        void* stream) {
  if (nv < 0 || b < 0 || (b > 0 && (!d_src || !d_dst || !d_dup)) || !d_offsets)
    return fail(TC_ERR_INVALID_ARG, "invalid batch arguments");
  if (b > (int64_t)INT32_MAX / 2) return fail(TC_ERR_CAPACITY, "batch too large");
  cudaStream_t s = (cudaStream_t)stream;
  uint64_t *k1 = nullptr, *k2 = nullptr;
  void* tmp = nullptr;
  size_t tb = 0;
  int32_t* cnt = nullptr;
  int64_t *off64 = nullptr, *tiles = nullptr;
  unsigned* err = nullptr;
  tc_status rc = TC_OK;
  unsigned herr = 0;
  do {
    if (::tc::dev_malloc(&k1, sizeof(uint64_t) * std::max<int64_t>(b, 1)) != cudaSuccess ||
        ::tc::dev_malloc(&k2, sizeof(uint64_t) * std::max<int64_t>(b, 1)) != cudaSuccess ||
        ::tc::dev_malloc(&cnt, sizeof(int32_t) * ((size_t)nv + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&off64, sizeof(int64_t) * ((size_t)nv + 2)) != cudaSuccess ||
        ::tc::dev_malloc(&tiles, sizeof(int64_t) * (size_t)(scan_tiles(nv) + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&err, sizeof(unsigned)) != cudaSuccess) {
      rc = fail(TC_ERR_OOM, "batch sort: allocation failed");
      break;
    }
    cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)nv + 1), s);
    cudaMemsetAsync(err, 0, sizeof(unsigned), s);
    if (b > 0) {
      k_pack_dir<<<grid_for(b, kThreads), kThreads, 0, s>>>(d_src, d_dst, b, k1);
      cub::DeviceRadixSort::SortKeys(nullptr, tb, k1, k2, (int)b, 0, 64, s);
      if (::tc::dev_malloc(&tmp, std::max<size_t>(tb, 1)) != cudaSuccess) {
        rc = fail(TC_ERR_OOM, "batch sort: allocation failed");
        break;
      }
      cub::DeviceRadixSort::SortKeys(tmp, tb, k1, k2, (int)b, 0, 64, s);
      k_unpack_dir<<<grid_for(b, kThreads), kThreads, 0, s>>>(k2, b, nv, d_src, d_dst, d_dup, cnt, err);
    }
    rc = scan_counts(cnt, nv, off64, tiles, s);
    if (rc != TC_OK) break;
    k_to_int32<<<grid_for((int64_t)nv + 1, kThreads), kThreads, 0, s>>>(off64, nv, d_offsets);
    cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = fail(TC_ERR_CUDA, "batch sort: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    if (herr) rc = fail(TC_ERR_INVALID_ARG, "batch has vertex ids outside [0, %d)", nv);
  } while (0);
  cudaFree(k1); cudaFree(k2); cudaFree(tmp); cudaFree(cnt); cudaFree(off64); cudaFree(tiles); cudaFree(err);
  return rc;
}

tc_status tc_insert_sorted(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, int64_t b, int32_t* d_dup,
                           int64_t* not_fitting, void* stream) {
  if (!g || b < 0 || (b > 0 && (!d_src || !d_dst || !d_dup))) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  cudaStream_t s = (cudaStream_t)stream;
  TC_TRY(ensure_stream_ws(g, (b + 1) / 2 + 1));
  StreamWs& w = *g->sw;
  TC_CUDA_TRY(cudaMemsetAsync(w.st, 0, sizeof(BatchStatus), s));
  if (not_fitting) *not_fitting = 0;
  if (b == 0) return TC_OK;
  SlackView view{g->start, g->used, g->pool};
  // entries come sorted by (src, dst): the packed keys of the new ones stay sorted, sentinel
  // elsewhere; sort once more to push the sentinels to the end.
  k_flag_present<<<grid_for(b, kThreads), kThreads, 0, s>>>(view, d_src, d_dst, d_dup, b, w.dk);
  size_t tb = w.cub_bytes;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortKeys(w.cub_tmp, tb, w.dk, w.dk2, (int)b, 0, 64, s));
  k_dir_runs<<<grid_for(b, kThreads), kThreads, 0, s>>>(w.dk2, b, g->used, g->cap, g->slack_q10, w.run_start, w.long_runs, w.long_cnt, w.st);
  TC_CUDA_TRY(cudaMemcpyAsync(w.st_host, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaMemcpyAsync(&w.st_host->pool_top, g->d_pool_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaStreamSynchronize(s));
  const BatchStatus h = *w.st_host;
  g->pool_top = (int64_t)h.pool_top;
  TC_TRY(ensure_pool(g, (int64_t)h.demand, s));
  if (h.n_runs > 0) {
    k_insert_runs<<<grid_for((int64_t)h.n_runs * 32, kThreads), kThreads, 0, s>>>(
        w.dk2, b, w.run_start, g->start, g->used, g->cap, g->pool, g->pool_cap, nullptr, w.ins_slot, g->d_pool_top,
        g->slack_q10, w.st);
    long_insert(g, w, b, nullptr, s);
    TC_CUDA_TRY(cudaGetLastError());
  }
  TC_CUDA_TRY(cudaMemcpyAsync(w.st_host, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaStreamSynchronize(s));
  if (w.st_host->err & (kErrPool | kErrScratch)) return fail(TC_ERR_CAPACITY, "adjacency pool or insertion scratch exhausted");
  g->m += (int64_t)w.st_host->dir_added;
  g->pool_top += (int64_t)h.demand;  // host bound until the next read of the device counter
  g->view_version++;
  if (not_fitting) *not_fitting = (int64_t)w.st_host->not_fitting;
  return TC_OK;
}

tc_status tc_delete_sorted(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, const int32_t* d_dup, int64_t b,
                           void* stream) {
  if (!g || b < 0 || (b > 0 && (!d_src || !d_dst || !d_dup))) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  cudaStream_t s = (cudaStream_t)stream;
  TC_TRY(ensure_stream_ws(g, (b + 1) / 2 + 1));
  TC_TRY(ensure_long_scratch(g));
  StreamWs& w = *g->sw;
  TC_CUDA_TRY(cudaMemsetAsync(w.st, 0, sizeof(BatchStatus), s));
  if (b == 0) return TC_OK;
  TC_CUDA_TRY(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), s));
  SlackView view{g->start, g->used, g->pool};
  k_mark_dir_deletions<<<grid_for(b, kThreads), kThreads, 0, s>>>(view, d_src, d_dst, d_dup, b, g->mark, w.first_del,
                                                                   w.vlist, w.counter);
  k_bump_epoch<<<1, 32, 0, s>>>(w.d_epoch);
  k_compact_marked<<<grid_for(b * 32, kThreads), kThreads, 0, s>>>(w.vlist, b, 1, w.counter, g->start, g->used,
                                                                   g->pool, g->mark, w.claim, w.d_epoch, w.first_del,
                                                                   w.st);
  long_compact(g, w, w.vlist, b, 1, w.counter, b, s);
  TC_CUDA_TRY(cudaGetLastError());
  TC_CUDA_TRY(cudaMemcpyAsync(w.st_host, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaStreamSynchronize(s));
  g->m -= (int64_t)w.st_host->dir_removed;
  g->view_version++;
  return TC_OK;
}

tc_status tc_count_batch(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, const int32_t* d_offsets,
                         const int32_t* d_dup, int64_t b, int sign, int32_t* per_vertex, int64_t* delta_dev,
                         const tc_sched* sched, void* stream) {
  tc::TraceRange trace_range("tc_count_batch");
  if (!g || b < 0 || (b > 0 && (!d_src || !d_dst || !d_dup || !d_offsets)) || (sign != 1 && sign != -1) || !per_vertex)
    return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  cudaStream_t s = (cudaStream_t)stream;
  TC_TRY(ensure_stream_ws(g, 1));
  StreamWs& w = *g->sw;
  TC_CUDA_TRY(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), s));
  if (b > 0) {
    DeltaArgs A = delta_args(g, to_params(sched));
    A.bl = BatchLists{d_src, d_dst, d_offsets, d_dup};
    A.count_host = b;
    A.sign = sign;
    A.weight = 1;
    A.only_present = sign < 0;
    A.split_items = w.split_items;
    A.split_cnt = &w.st->n_split[0];
    TC_CUDA_TRY(cudaMemsetAsync(A.split_cnt, 0, sizeof(unsigned long long), s));
    k_delta<kPredBatch><<<delta_grid(), kThreads, delta_smem(A), s>>>(A, reinterpret_cast<uint32_t*>(per_vertex),
                                                                     w.counter);
    k_delta_split<kPredBatch><<<delta_grid(), kThreads, delta_smem(A), s>>>(A, reinterpret_cast<uint32_t*>(per_vertex),
                                                                           w.counter);
    TC_CUDA_TRY(cudaGetLastError());
  }
  if (delta_dev) {
    if (sign > 0) k_add_delta<<<1, 32, 0, s>>>(delta_dev, w.counter, nullptr);
    else k_add_delta<<<1, 32, 0, s>>>(delta_dev, nullptr, w.counter);
    TC_CUDA_TRY(cudaGetLastError());
  }
  return TC_OK;
}

}  // extern "C"

// ---- captured streaming pipeline ---------------------------------------------------------------
//
// tc_apply_batch reads the batch's sizes and the pool demand on the host halfway through (one
// synchronisation) and sizes each launch from them. The pipeline below runs the same steps as
// one CUDA graph per batch-size bin instead: every launch is sized for the bin's capacity and
// reads the batch's real counts from device memory (grid-stride loops over device counts, the
// batch padded with sentinel keys), so a batch is one small launch that loads it and its size
// into the bin's buffers (k_load_batch) and one graph launch, with no host synchronisation
// inside. The delta count of each phase (deletions, insertions) is one
// persistent kernel (k_delta_fused). The pool headroom the relocations of one batch can take is
// bounded ahead (every touched list moving: (m + 2b)(1 + slack) slots) and reserved before the
// launch, so the device bump allocator cannot run out. The graphs capture the graph's pool and
// workspace pointers and the caller's per-vertex and delta arrays; they are captured again when
// any of these change.
//
// Autotuner (tc_pipeline_autotune): the bins start as a fine ladder of capacities (2^10, 2^11,
// ... up to max_batch). Over the next k batches each batch runs under one "arm" of its natural
// bin (the smallest that holds it): one of the candidate tile shapes of the delta kernel (CTAs
// per SM, split threshold and split-item size) in that bin's graph, or the default shape in the
// next bin's graph. Each arm's time per update is measured with events. At the end every bin
// keeps its fastest shape, and a bin whose batches ran no more than 3 % slower in the next bin's
// graph is merged into it: its threshold is dropped and its batches use that graph (fewer
// graphs where padding costs nothing, the fine ladder where it does).

namespace tc {
namespace {
constexpr int kPipeBins = 16;
constexpr int64_t kPipeMinBin = 1 << 10;
struct PipeCand {
  int ctas;       // persistent delta kernel CTAs per SM (0 = the occupancy limit)
  int chunk;      // split-item size: entries of the shorter list
  int split_min;  // intersections whose shorter list is longer than this are split
};
constexpr int kPipeCands = 5;
constexpr PipeCand kPipeCand[kPipeCands] = {
    {0, kDeltaChunk, kDeltaSplit}, {0, kDeltaChunk / 2, kDeltaSplit / 2}, {0, kDeltaChunk / 4, kDeltaSplit / 4},
    {0, kDeltaChunk / 8, kDeltaSplit / 8}, {0, kDeltaChunk / 16, kDeltaSplit / 16}};
constexpr int kPipeArms = kPipeCands + 1;  // + the default shape in the next bin's graph
constexpr double kMergeSlack = 1.03;
}  // namespace
}  // namespace tc

struct tc_pipeline {
  tc_graph* g = nullptr;
  int device = -1;
  int64_t b_max = 0;
  int nbins = 0;
  int64_t bin_cap[tc::kPipeBins] = {};
  int cand[tc::kPipeBins] = {};                      // chosen tile-shape candidate per bin
  int serve[tc::kPipeBins] = {};                     // bin whose graph runs this bin's batches
  cudaGraphExec_t exec[tc::kPipeBins][tc::kPipeCands] = {};
  // autotuning: per natural bin and arm, accumulated ms per update and samples
  double tune_ms_per_update[tc::kPipeBins][tc::kPipeArms] = {};
  int tune_n[tc::kPipeBins][tc::kPipeArms] = {};
  int tune_left = 0;                                 // batches still spent exploring
  // what the captured graphs hold
  const void* key_pool = nullptr;
  const void* key_mark = nullptr;
  const void* key_pv = nullptr;
  const void* key_delta = nullptr;
  uint64_t key_ws = 0;
  int64_t key_pool_cap = 0;
  tc::SchedParams sp;
  unsigned long long spin_ns = tc::kSpinNs;          // bound of the delta kernel's barrier wait
  unsigned bar_extra = 0;                            // (test hook: arrivals that never come)
  cudaStream_t cs = nullptr;     // capture stream
  int64_t* d_b = nullptr;
  tc::BatchStatus* h_st = nullptr;          // pinned: status of the last batch
  unsigned long long* h_top = nullptr;      // pinned: pool bump pointer after it
  uint32_t* pv_scratch = nullptr;
  int64_t* delta_scratch = nullptr;
  cudaEvent_t done = nullptr, t0 = nullptr, t1 = nullptr;
  cudaEvent_t pev[4] = {};       // profiling: around the two delta kernels, inside the graphs
  bool profile = false;
  int64_t prof_batches = 0;
  double prof_delta_ms = 0.0;
  int64_t prof_delta_bytes = 0;
  bool pending = false;
  int pending_bin = -1, pending_cand = -1, pending_arm = -1, pending_nat = -1;
  int64_t pending_b = 0;
  bool timing = false;
  tc_batch_info last{};
};

namespace tc {
namespace {

void drop_graphs(tc_pipeline* p) {
  for (int i = 0; i < kPipeBins; ++i)
    for (int j = 0; j < kPipeCands; ++j)
      if (p->exec[i][j]) {
        cudaGraphExecDestroy(p->exec[i][j]);
        p->exec[i][j] = nullptr;
      }
}

// Fold the finished batch's device status into the host view of the graph.
tc_status pipe_settle(tc_pipeline* p) {
  if (!p->pending) return TC_OK;
  TC_CUDA_TRY(cudaEventSynchronize(p->done));
  p->pending = false;
  tc_graph* g = p->g;
  const BatchStatus& f = *p->h_st;
  g->pool_top = (int64_t)*p->h_top;
  g->m += 2 * ((int64_t)f.n_ins - (int64_t)f.n_del);
  g->view_version++;
  p->last.updates = p->pending_b;
  p->last.inserted = (int64_t)f.n_ins;
  p->last.deleted = (int64_t)f.n_del;
  p->last.ignored = p->pending_b - (int64_t)f.n_ins - (int64_t)f.n_del;
  p->last.triangles_added = (int64_t)f.tri_added;
  p->last.triangles_removed = (int64_t)f.tri_removed;
  p->last.status = TC_OK;
  if (p->timing) {
    float ms = 0.f;
    TC_CUDA_TRY(cudaEventElapsedTime(&ms, p->t0, p->t1));
    const int bi = p->pending_nat, a = p->pending_arm;
    p->tune_ms_per_update[bi][a] += (double)ms / (double)std::max<int64_t>(p->pending_b, 1);
    p->tune_n[bi][a] += 1;
    p->timing = false;
  }
  if (p->profile && p->prof_delta_ms >= 0.0) {
    // a failed read (no event recorded by the graph) turns the profile off, not the batch
    float d0 = 0.f, d1 = 0.f;
    if (cudaEventElapsedTime(&d0, p->pev[0], p->pev[1]) != cudaSuccess ||
        cudaEventElapsedTime(&d1, p->pev[2], p->pev[3]) != cudaSuccess) {
      cudaGetLastError();
      p->prof_delta_ms = -1.0;
    } else {
      p->prof_batches += 1;
      p->prof_delta_ms += (double)d0 + (double)d1;
      p->prof_delta_bytes += (int64_t)f.delta_bytes;
    }
  }
  if (f.err & kErrRange) {
    p->last.status = TC_ERR_INVALID_ARG;
    return fail(TC_ERR_INVALID_ARG, "batch had vertex ids outside [0, %d); they were ignored", g->n);
  }
  if (f.err & (kErrPool | kErrScratch)) {
    p->last.status = TC_ERR_CAPACITY;
    return fail(TC_ERR_CAPACITY, "adjacency pool or insertion scratch exhausted");
  }
  if (f.err & kErrTimeout) {
    p->last.status = TC_ERR_TIMEOUT;
    return fail(TC_ERR_TIMEOUT, "the delta kernel gave up waiting for queued work; the batch's count is incomplete");
  }
  return TC_OK;
}

int64_t pipe_worst_demand(const tc_graph* g, int64_t b) {
  const int64_t q = std::max<int64_t>(g->slack_q10, 256);
  return ((g->m + 2 * b) * (1024 + q) + 1023) / 1024 + 16 * b + 64;
}

// Drop the captured graphs when what they hold (pool, marks, workspace, outputs) has changed.
void pipe_check_keys(tc_pipeline* p, const void* pv, const void* delta) {
  tc_graph* g = p->g;
  const StreamWs& w = *g->sw;
  if (p->key_pool != g->pool || p->key_mark != g->mark || p->key_pv != pv || p->key_delta != delta ||
      p->key_ws != w.version || p->key_pool_cap != g->pool_cap) {
    drop_graphs(p);
    p->key_pool = g->pool;
    p->key_mark = g->mark;
    p->key_pv = pv;
    p->key_delta = delta;
    p->key_ws = w.version;
    p->key_pool_cap = g->pool_cap;
  }
}

// Record the whole batch pipeline for a bin of capacity cap, with tile shape `cand`, on the
// capture stream.
tc_status pipe_capture(tc_pipeline* p, int bin, int cand, uint32_t* pv, int64_t* delta) {
  tc_graph* g = p->g;
  StreamWs& w = *g->sw;
  const int64_t cap = p->bin_cap[bin];
  const PipeCand& pc = kPipeCand[cand];
  cudaStream_t s = p->cs;
  const int L = bits_for(std::max(g->n, 2));
  const uint64_t sent = (1ull << (2 * L + 1)) - 1;
  const SlackView view{g->start, g->used, g->pool};
  const int gb = grid_for(cap, kThreads);
  const int g2 = grid_for(2 * cap, kThreads);
  const int gw = grid_for(2 * cap * 32, kThreads);
  int gdelta = 0, ghub = 0;
  const size_t dsm = delta_smem(delta_args(g, p->sp));
  TC_TRY(fused_grid(pc.ctas, dsm, &gdelta));
  TC_TRY(hub_grid(&ghub));
  cudaGraph_t graph = nullptr;
  TC_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  do {
    cudaMemsetAsync(w.st, 0, sizeof(BatchStatus), s);
    k_make_keys_cap<<<gb, kThreads, 0, s>>>(w.src, w.dst, w.isdel, p->d_b, cap, g->n, L, w.keys, w.st);
    size_t tb = w.cub_bytes;
    if ((e = cub::DeviceRadixSort::SortKeys(w.cub_tmp, tb, w.keys, w.keys2, (int)cap, 0, 2 * L + 1, s)) != cudaSuccess)
      break;
    k_run_heads<<<gb, kThreads, 0, s>>>(w.keys2, cap, sent, w.head);
    cudaMemsetAsync(w.dk, 0xff, sizeof(uint64_t) * 2 * cap, s);
    k_classify<<<gb, kThreads, 0, s>>>(view, w.keys2, cap, L, w.head, w.dlist, w.ilist, w.dk, w.st);
    size_t tb2 = w.cub_bytes;
    if ((e = cub::DeviceRadixSort::SortKeys(w.cub_tmp, tb2, w.dk, w.dk2, (int)(2 * cap), 0, 64, s)) != cudaSuccess)
      break;
    k_dir_runs<<<g2, kThreads, 0, s>>>(w.dk2, 2 * cap, g->used, g->cap, g->slack_q10, w.run_start, w.long_runs, w.long_cnt, w.st);
    // deletions: mark, count on the pre-deletion graph, compact
    k_mark_deletions<<<gb, kThreads, 0, s>>>(w.dlist, w.st, g->start, g->mark, w.first_del);
    DeltaArgs A = delta_args(g, p->sp);
    A.dlist = w.dlist;
    A.count_dev = &w.st->n_del;
    A.sign = -1;
    A.weight = 2;
    A.chunk = pc.chunk;
    A.split_min = pc.split_min;
    A.spin_ns = p->spin_ns;
    A.bar_extra = p->bar_extra;
    A.split_items = w.split_items;
    A.split_cnt = &w.st->n_split[0];
    A.entry_done = &w.st->entry_done[0];
    A.item_tag = w.item_tag;
    A.item_epoch = w.item_epoch;
    A.err = &w.st->err;
    A.bytes_out = &w.st->delta_bytes;
    A.e_next = &w.st->e_next[0];
    A.i_next = &w.st->i_next[0];
    if (p->profile) cudaEventRecordWithFlags(p->pev[0], s, cudaEventRecordExternal);
    hub_kernels(A, w, 0, cap, ghub, pv, &w.st->tri_removed, s);
    k_bump_epoch<<<1, 32, 0, s>>>(w.item_epoch);
    k_delta_fused<kPredMark><<<gdelta, kThreads, dsm, s>>>(A, pv, &w.st->tri_removed);
    if (p->profile) cudaEventRecordWithFlags(p->pev[1], s, cudaEventRecordExternal);
    k_endpoints<<<gb, kThreads, 0, s>>>(w.dlist, w.st, w.vlist);
    k_bump_epoch<<<1, 32, 0, s>>>(w.d_epoch);
    k_compact_marked<<<gw, kThreads, 0, s>>>(w.vlist, 0, 2, &w.st->n_del, g->start, g->used, g->pool, g->mark,
                                             w.claim, w.d_epoch, w.first_del, w.st);
    long_compact(g, w, w.vlist, 0, 2, &w.st->n_del, 2 * cap, s);
    // insertions: merge, count on the post-insertion graph, clear the marks
    k_insert_runs<<<gw, kThreads, 0, s>>>(w.dk2, 2 * cap, w.run_start, g->start, g->used, g->cap, g->pool,
                                          g->pool_cap, g->mark, w.ins_slot, g->d_pool_top, g->slack_q10, w.st);
    long_insert(g, w, 2 * cap, g->mark, s);
    DeltaArgs B = A;
    B.dlist = nullptr;
    B.ilist = w.ilist;
    B.count_dev = &w.st->n_ins;
    B.sign = 1;
    B.split_cnt = &w.st->n_split[1];
    B.entry_done = &w.st->entry_done[1];
    B.e_next = &w.st->e_next[1];
    B.i_next = &w.st->i_next[1];
    if (p->profile) cudaEventRecordWithFlags(p->pev[2], s, cudaEventRecordExternal);
    hub_kernels(B, w, 1, cap, ghub, pv, &w.st->tri_added, s);
    k_bump_epoch<<<1, 32, 0, s>>>(w.item_epoch);
    k_delta_fused<kPredMark><<<gdelta, kThreads, dsm, s>>>(B, pv, &w.st->tri_added);
    if (p->profile) cudaEventRecordWithFlags(p->pev[3], s, cudaEventRecordExternal);
    k_clear_slots<<<g2, kThreads, 0, s>>>(w.ins_slot, 0, &w.st->n_ins, g->mark);
    k_add_delta<<<1, 32, 0, s>>>(delta, &w.st->tri_added, &w.st->tri_removed);
    cudaMemcpyAsync(p->h_st, w.st, sizeof(BatchStatus), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(p->h_top, g->d_pool_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    e = cudaGetLastError();
  } while (0);
  const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec[bin][cand], graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    p->exec[bin][cand] = nullptr;
    return fail(TC_ERR_CUDA, "pipeline capture: %s", cudaGetErrorString(e));
  }
  return TC_OK;
}

// End of the exploration: the fastest shape per bin, then the merges (top bin down, so a chain
// of merged bins resolves to the graph that serves the highest of them).
void pipe_finish_tuning(tc_pipeline* p) {
  for (int i = 0; i < p->nbins; ++i) {
    int best = p->cand[i];
    double best_v = 0.0;
    for (int j = 0; j < kPipeCands; ++j) {
      if (p->tune_n[i][j] < 1) continue;
      const double v = p->tune_ms_per_update[i][j] / p->tune_n[i][j];
      if (best_v == 0.0 || v < best_v) {
        best_v = v;
        best = j;
      }
    }
    p->cand[i] = best;
  }
  p->serve[p->nbins - 1] = p->nbins - 1;
  for (int i = p->nbins - 2; i >= 0; --i) {
    p->serve[i] = i;
    const int own = 0, up = kPipeCands;
    if (p->tune_n[i][own] > 0 && p->tune_n[i][up] > 0) {
      const double v_own = p->tune_ms_per_update[i][own] / p->tune_n[i][own];
      const double v_up = p->tune_ms_per_update[i][up] / p->tune_n[i][up];
      if (v_up <= kMergeSlack * v_own) p->serve[i] = p->serve[i + 1];
    }
  }
}

int pipe_natural_bin(const tc_pipeline* p, int64_t b) {
  int bin = 0;
  while (bin + 1 < p->nbins && p->bin_cap[bin] < b) ++bin;
  return bin;
}

}  // namespace
}  // namespace tc

extern "C" {

tc_status tc_pipeline_create(tc_graph* g, int64_t max_batch, const tc_sched* sched, tc_pipeline** out) {
  if (!g || !out || max_batch < 1) return fail(TC_ERR_INVALID_ARG, "invalid pipeline arguments");
  if (max_batch > (int64_t)INT32_MAX / 4) return fail(TC_ERR_CAPACITY, "pipeline batch capacity exceeds 2^29");
  *out = nullptr;
  tc_pipeline* p = new tc_pipeline();
  p->g = g;
  p->sp = to_params(sched);
  TC_CUDA_TRY(cudaGetDevice(&p->device));
  // fine ladder: 2^10, 2^11, ... (the last bin holds max_batch; past kPipeBins bins the ladder
  // doubles its step)
  int64_t step = 2;
  {
    int64_t levels = 1;
    for (int64_t c = kPipeMinBin; c < max_batch; c *= 2) ++levels;
    while (levels > kPipeBins) {
      step *= 2;
      levels = (levels + 1) / 2;
    }
  }
  for (int64_t c = kPipeMinBin; p->nbins < kPipeBins; c *= step) {
    p->bin_cap[p->nbins++] = std::min(c, std::max(max_batch, kPipeMinBin));
    if (c >= max_batch) break;
  }
  p->b_max = p->bin_cap[p->nbins - 1];
  for (int i = 0; i < kPipeBins; ++i) {
    p->cand[i] = 0;
    p->serve[i] = i;
  }
  tc_status rc = TC_OK;
  do {
    if ((rc = ensure_stream_ws(g, p->b_max)) != TC_OK) break;
    if (cudaStreamCreateWithFlags(&p->cs, cudaStreamNonBlocking) != cudaSuccess ||
        ::tc::dev_malloc(&p->d_b, sizeof(int64_t)) != cudaSuccess ||
        cudaMallocHost(&p->h_st, sizeof(BatchStatus)) != cudaSuccess ||
        cudaMallocHost(&p->h_top, sizeof(unsigned long long)) != cudaSuccess ||
        ::tc::dev_malloc(&p->pv_scratch, sizeof(uint32_t) * ((size_t)g->n + 1)) != cudaSuccess ||
        ::tc::dev_malloc(&p->delta_scratch, sizeof(int64_t)) != cudaSuccess ||
        cudaEventCreate(&p->done) != cudaSuccess || cudaEventCreate(&p->t0) != cudaSuccess ||
        cudaEventCreate(&p->t1) != cudaSuccess || cudaEventCreate(&p->pev[0]) != cudaSuccess ||
        cudaEventCreate(&p->pev[1]) != cudaSuccess || cudaEventCreate(&p->pev[2]) != cudaSuccess ||
        cudaEventCreate(&p->pev[3]) != cudaSuccess) {
      rc = fail(TC_ERR_OOM, "pipeline: allocation failed");
      break;
    }
    if (cudaMemset(p->pv_scratch, 0, sizeof(uint32_t) * ((size_t)g->n + 1)) != cudaSuccess ||
        cudaMemset(p->delta_scratch, 0, sizeof(int64_t)) != cudaSuccess)
      rc = fail(TC_ERR_CUDA, "pipeline: set-up failed");
  } while (0);
  if (rc != TC_OK) {
    tc_pipeline_destroy(p);
    return rc;
  }
  *out = p;
  return TC_OK;
}

tc_status tc_pipeline_destroy(tc_pipeline* p) {
  if (!p) return TC_OK;
  if (p->pending) cudaEventSynchronize(p->done);
  drop_graphs(p);
  if (p->cs) cudaStreamDestroy(p->cs);
  cudaFree(p->d_b);
  cudaFreeHost(p->h_st);
  cudaFreeHost(p->h_top);
  cudaFree(p->pv_scratch);
  cudaFree(p->delta_scratch);
  if (p->done) cudaEventDestroy(p->done);
  if (p->t0) cudaEventDestroy(p->t0);
  if (p->t1) cudaEventDestroy(p->t1);
  for (int i = 0; i < 4; ++i)
    if (p->pev[i]) cudaEventDestroy(p->pev[i]);
  delete p;
  return TC_OK;
}

tc_status tc_pipeline_apply(tc_pipeline* p, const int32_t* d_src, const int32_t* d_dst, const uint8_t* d_is_delete,
                            int64_t b, int32_t* per_vertex, int64_t* delta_dev, void* stream) {
  tc::TraceRange trace_range("tc_pipeline_apply");
  if (!p || b < 0 || (b > 0 && (!d_src || !d_dst))) return fail(TC_ERR_INVALID_ARG, "invalid batch arguments");
  if (b > p->b_max)
    return fail(TC_ERR_CAPACITY, "batch of %lld updates exceeds the pipeline's %lld", (long long)b,
                (long long)p->b_max);
  int dev = 0;
  TC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != p->device) return fail(TC_ERR_INVALID_ARG, "pipeline used on device %d, created on %d", dev, p->device);
  TC_TRY(pipe_settle(p));
  tc_graph* g = p->g;
  cudaStream_t s = (cudaStream_t)stream;
  if (b == 0) return TC_OK;
  // Headroom for the worst case: every list the batch touches moves to the pool top.
  const int64_t worst = pipe_worst_demand(g, b);
  if (g->pool_cap - g->pool_top < worst) TC_TRY(ensure_pool(g, worst + worst / 2, s));
  TC_TRY(ensure_stream_ws(g, p->b_max));
  TC_TRY(ensure_long_scratch(g));
  uint32_t* pv = per_vertex ? reinterpret_cast<uint32_t*>(per_vertex) : p->pv_scratch;
  int64_t* delta = delta_dev ? delta_dev : p->delta_scratch;
  StreamWs& w = *g->sw;
  pipe_check_keys(p, pv, delta);
  const int nat = pipe_natural_bin(p, b);
  int bin = p->serve[nat];
  int cand = p->cand[bin];
  int arm = -1;
  if (p->tune_left > 0) {
    // explore: the arm of this natural bin with the fewest samples
    arm = 0;
    const int narms = nat + 1 < p->nbins ? kPipeArms : kPipeCands;
    for (int j = 1; j < narms; ++j)
      if (p->tune_n[nat][j] < p->tune_n[nat][arm]) arm = j;
    bin = arm < kPipeCands ? nat : nat + 1;
    cand = arm < kPipeCands ? arm : 0;
  }
  if (!p->exec[bin][cand]) TC_TRY(pipe_capture(p, bin, cand, pv, delta));
  // the batch into the capacity-sized buffers the graph reads, and its size
  k_load_batch<<<grid_for(b, kThreads), kThreads, 0, s>>>(d_src, d_dst, d_is_delete, b, w.src, w.dst, w.isdel,
                                                         p->d_b);
  TC_CUDA_TRY(cudaGetLastError());
  p->timing = arm >= 0;
  if (p->timing) TC_CUDA_TRY(cudaEventRecord(p->t0, s));
  TC_CUDA_TRY(cudaGraphLaunch(p->exec[bin][cand], s));
  if (p->timing) TC_CUDA_TRY(cudaEventRecord(p->t1, s));
  TC_CUDA_TRY(cudaEventRecord(p->done, s));
  p->pending = true;
  p->pending_bin = bin;
  p->pending_cand = cand;
  p->pending_arm = arm;
  p->pending_nat = nat;
  p->pending_b = b;
  if (p->tune_left > 0 && --p->tune_left == 0) {
    // exploration over: settle the last sample, keep the fastest shape per bin, merge bins
    TC_TRY(pipe_settle(p));
    pipe_finish_tuning(p);
  }
  return TC_OK;
}

tc_status tc_pipeline_prepare(tc_pipeline* p, int32_t* per_vertex, int64_t* delta_dev, void* stream) {
  if (!p) return fail(TC_ERR_INVALID_ARG, "pipeline is NULL");
  TC_TRY(pipe_settle(p));
  tc_graph* g = p->g;
  const int64_t worst = pipe_worst_demand(g, p->b_max);
  if (g->pool_cap - g->pool_top < worst) TC_TRY(ensure_pool(g, 2 * worst, (cudaStream_t)stream));
  TC_TRY(ensure_stream_ws(g, p->b_max));
  TC_TRY(ensure_long_scratch(g));
  uint32_t* pv = per_vertex ? reinterpret_cast<uint32_t*>(per_vertex) : p->pv_scratch;
  int64_t* delta = delta_dev ? delta_dev : p->delta_scratch;
  pipe_check_keys(p, pv, delta);
  for (int i = 0; i < p->nbins; ++i) {
    const int bin = p->serve[i];
    if (!p->exec[bin][p->cand[bin]]) TC_TRY(pipe_capture(p, bin, p->cand[bin], pv, delta));
  }
  return TC_OK;
}

tc_status tc_pipeline_sync(tc_pipeline* p, tc_batch_info* last) {
  if (!p) return fail(TC_ERR_INVALID_ARG, "pipeline is NULL");
  TC_TRY(pipe_settle(p));
  if (last) *last = p->last;
  return TC_OK;
}

tc_status tc_pipeline_autotune(tc_pipeline* p, int32_t batches) {
  if (!p || batches < 0) return fail(TC_ERR_INVALID_ARG, "invalid autotune arguments");
  TC_TRY(pipe_settle(p));
  memset(p->tune_ms_per_update, 0, sizeof(p->tune_ms_per_update));
  memset(p->tune_n, 0, sizeof(p->tune_n));
  for (int i = 0; i < kPipeBins; ++i) p->serve[i] = i;
  p->tune_left = batches;
  return TC_OK;
}

tc_status tc_pipeline_info(const tc_pipeline* p, int32_t* nbins, int64_t* bin_cap, int32_t* delta_blocks_per_sm) {
  if (!p) return fail(TC_ERR_INVALID_ARG, "pipeline is NULL");
  if (nbins) *nbins = p->nbins;
  for (int i = 0; i < p->nbins; ++i) {
    const int bin = p->serve[i];
    if (bin_cap) bin_cap[i] = p->bin_cap[i];
    if (delta_blocks_per_sm) {
      int grid = 0;
      if (fused_grid(kPipeCand[p->cand[bin]].ctas, delta_smem(delta_args(p->g, p->sp)), &grid) != TC_OK)
        return TC_ERR_CUDA;
      delta_blocks_per_sm[i] = grid / device_info().sms;
    }
  }
  return TC_OK;
}

tc_status tc_pipeline_plan_get(const tc_pipeline* p, tc_pipeline_plan* plan) {
  if (!p || !plan) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  memset(plan, 0, sizeof(*plan));
  plan->nbins = p->nbins;
  for (int i = 0; i < p->nbins; ++i) {
    const PipeCand& c = kPipeCand[p->cand[p->serve[i]]];
    plan->bin_cap[i] = p->bin_cap[i];
    plan->serve[i] = p->serve[i];
    plan->ctas_per_sm[i] = c.ctas;
    plan->chunk[i] = c.chunk;
    plan->split_min[i] = c.split_min;
  }
  return TC_OK;
}

tc_status tc_pipeline_plan_set(tc_pipeline* p, const tc_pipeline_plan* plan) {
  if (!p || !plan) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  if (plan->nbins != p->nbins) return fail(TC_ERR_INVALID_ARG, "plan has %d bins, the pipeline %d", plan->nbins, p->nbins);
  int cand[kPipeBins], serve[kPipeBins];
  for (int i = 0; i < p->nbins; ++i) {
    if (plan->bin_cap[i] != p->bin_cap[i]) return fail(TC_ERR_INVALID_ARG, "plan bin %d capacity differs", i);
    if (plan->serve[i] < i || plan->serve[i] >= p->nbins || (i > 0 && plan->serve[i] < plan->serve[i - 1]))
      return fail(TC_ERR_INVALID_ARG, "plan bin %d is served by bin %d", i, plan->serve[i]);
    cand[i] = -1;
    for (int j = 0; j < kPipeCands; ++j)
      if (kPipeCand[j].ctas == plan->ctas_per_sm[i] && kPipeCand[j].chunk == plan->chunk[i] &&
          kPipeCand[j].split_min == plan->split_min[i])
        cand[i] = j;
    if (cand[i] < 0) return fail(TC_ERR_INVALID_ARG, "plan bin %d: tile shape is not one of the candidates", i);
    serve[i] = plan->serve[i];
  }
  TC_TRY(pipe_settle(p));
  for (int i = 0; i < p->nbins; ++i) {
    p->serve[i] = serve[i];
    p->cand[serve[i]] = cand[i];
  }
  p->tune_left = 0;
  return TC_OK;
}

tc_status tc_pipeline_profile(tc_pipeline* p, int on) {
  if (!p) return fail(TC_ERR_INVALID_ARG, "pipeline is NULL");
  TC_TRY(pipe_settle(p));
  if ((on != 0) != p->profile) drop_graphs(p);  // the event records live inside the graphs
  p->profile = on != 0;
  p->prof_batches = 0;
  p->prof_delta_ms = 0.0;
  p->prof_delta_bytes = 0;
  return TC_OK;
}

tc_status tc_pipeline_stats(tc_pipeline* p, int64_t* batches, double* delta_ms, int64_t* delta_bytes) {
  if (!p) return fail(TC_ERR_INVALID_ARG, "pipeline is NULL");
  TC_TRY(pipe_settle(p));
  if (batches) *batches = p->prof_batches;
  if (delta_ms) *delta_ms = p->prof_delta_ms;
  if (delta_bytes) *delta_bytes = p->prof_delta_bytes;
  return TC_OK;
}

tc_status tc_pipeline_set_wait_bound(tc_pipeline* p, uint64_t wait_ns, int32_t extra_arrivals) {
  if (!p || wait_ns == 0 || extra_arrivals < 0) return fail(TC_ERR_INVALID_ARG, "invalid wait bound");
  TC_TRY(pipe_settle(p));
  p->spin_ns = wait_ns;
  p->bar_extra = (unsigned)extra_arrivals;
  drop_graphs(p);  // the bound is an argument of the captured launches
  return TC_OK;
}

}  // extern "C"
