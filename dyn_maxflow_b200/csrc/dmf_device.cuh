// dmf_device.cuh -- device-side building blocks of the sm_100a solver:
// memory-order helpers, the bounded grid barrier, queue appends and the group
// abstractions (a warp tile or a whole block working on one vertex).
#pragma once

#include <climits>
#include <cstdint>
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

namespace dmfd {

namespace cg = cooperative_groups;

// ---- error bits (Ctrl::err) ------------------------------------------------
enum : int {
  ERR_TIMEOUT = 1,       // a grid-barrier wait ran out of time
  ERR_NO_CONV = 2,       // outer-iteration bound reached
  ERR_UNKNOWN_ARC = 4,   // update names an absent arc
  ERR_DUP_ARC = 8,       // arc twice in one batch
  ERR_BAD_UPDATE = 16,   // vertex id out of range or capacity out of bounds
};

// Barrier wait limit: 4 s of %globaltimer.  Any single phase of a solve is
// orders of magnitude shorter; hitting it means a block never arrived.
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;
// The limit under the failure-injection test hook (DMF_FLAG_TEST_BARRIER_TIMEOUT).
constexpr unsigned long long kTestBarrierTimeoutNs = 20000000ull;

// Per-phase counters, triple-buffered: phase k appends into slot k%3, reads
// slot (k-1)%3, and block 0 clears slot (k+1)%3.
struct Slot {
  int q;             // normal-queue tail
  int hq;            // hub-queue tail
  long long arcs;    // sum of degrees of appended vertices
  int cnt;           // generic counter (BFS: active vertices labelled; topo push: active seen)
  int pad;
};

// Control block of one solver (device memory, cleared before every launch).
struct Ctrl {
  unsigned int bar_count;     // grid barrier: arrivals (low bits) and generation (top bit)
  unsigned int bar_gen;       // unused
  int err;
  int err_info;
  Slot slot[3];
  // per global relabel
  int act_q, act_hq;          // active list tails built by the BFS
  int pos_count;              // vertices with excess > 0 (not s, t, dead)
  int pad0;
  long long unexplored;       // arcs of not-yet-labelled candidate vertices
  long long flow;             // result
  // statistics
  unsigned long long st_outer, st_levels, st_rounds, st_pushes, st_relabels, st_arcs, st_visits, st_dead;
  unsigned int rounds_used;
  int trace_len;              // entries written to the optional timeline
  // push-round worklist tails and topology-driven active counts, round r uses [r % 3]
  int wtail[3], whtail[3], seen[3];
  int pad1;
  unsigned long long probe[2];  // longest work item of a phase, (ns << 32) | vertex
  unsigned long long blk[2];    // longest block work of a phase (ns), barrier exit to arrival
  // kept dead set (dynamic batches): vertices of the dead set whose excess a batch
  // lowered or that a pull moved a deficit to (candidates for deficits), the
  // deficits found among them, and those left after the local repair
  int dcand;
  int dseeds;
  long long dneed;
  int dleft;
  int dkept;                    // 1: the dead set was kept for the global relabels
  unsigned long long st_barcs;  // adjacency entries read by global-relabel BFS levels
  unsigned long long st_dseeds; // deficits inside the kept dead set (first local pass)
  unsigned long long st_revived; // dead vertices revived because they reach a deficit left over
  int dup_at;                   // 1 + an update whose arc an earlier update of the batch names (0: none)
  int nreopen;                  // updates queued for reopening (kept dead set)
  int nrepair;                  // updates queued for the over-capacity repair
  int pad3;
};

// ---- memory helpers ---------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_vol(const int *p) { return *(const volatile int *)p; }
__device__ __forceinline__ long long ld_vol(const long long *p) { return *(const volatile long long *)p; }
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ long long atomic_add_ll(long long *p, long long v) {
  return (long long)atomicAdd((unsigned long long *)p, (unsigned long long)v);
}

// ---- bounded grid barrier ---------------------------------------------------
// All blocks of a cooperative launch call it the same number of times.  Thread
// 0 of each block arrives with ONE atomic on bar_count: block 0 adds
// 2^31 - (G - 1), every other block adds 1, so the counter's top bit flips
// exactly when the last of the G blocks arrives (and the low bits return to
// where they were: nothing has to be reset between barriers).  A waiter polls
// until the top bit differs from the value its own arrival saw; a block that
// is already in the next barrier cannot flip it back, because that flip needs
// every block, the waiter included.  Polls check the error word and the
// %globaltimer limit (`limit_ns`, normally kBarrierTimeoutNs) every 64 iterations.
//
// After the wait, warp 0 copies the whole control block into `snap` (shared
// memory): the phase that follows reads the counters the previous phase
// produced from there, so a phase costs G control-block reads instead of one
// per warp on a single L2 line.  Returns false (uniformly per block) when an
// error is set.
__device__ __forceinline__ bool grid_barrier(Ctrl *c, Ctrl *snap, unsigned long long limit_ns) {
  __shared__ int s_err;
  __syncthreads();
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      const unsigned nb = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
      __threadfence();
      const unsigned old = atomicAdd(&c->bar_count, nb);
      unsigned long long t0 = 0;
      int spins = 0;
      while (((ld_acquire_u32(&c->bar_count) ^ old) & 0x80000000u) == 0) {
        __nanosleep(32);
        if ((++spins & 63) == 0) {
          if (ld_vol(&c->err)) break;
          const unsigned long long now = globaltimer();
          if (!t0) {
            t0 = now;
          } else if (now - t0 > limit_ns) {
            atomicOr(&c->err, ERR_TIMEOUT);
            break;
          }
        }
      }
      __threadfence();
    }
    __syncwarp();
    const int *src = (const int *)c;
    int *dst = (int *)snap;
    for (int w = threadIdx.x; w < (int)(sizeof(Ctrl) / 4); w += 32) dst[w] = __ldcg(src + w);
    __syncwarp();
    if (threadIdx.x == 0) s_err = snap->err;
  }
  __syncthreads();
  return s_err == 0;
}

// ---- work-item numbering ----------------------------------------------------
// Worklist items are numbered blocks first: thread t of block b is worker
// t * G + b (G blocks), so items 0 .. G-1 go to G different blocks -- every SM
// -- before any block takes a second one.  A short list (a BFS level on a
// grid, a push round late in a solve) is then worked on by all SMs at once
// instead of filling the first blocks, whose load/store units would serialise
// its scattered accesses.  Loops over every vertex keep the contiguous
// numbering, which keeps their per-vertex array accesses coalesced.
// `rot` rotates the order inside a block so that thread `rot` takes a block's
// first item: the kinds of work of one phase (hub chunks, one-thread items,
// tile items) start on different warps and run side by side when the lists are
// short, instead of queueing on warp 0.
__device__ __forceinline__ int spread_thread(int rot = 0) {
  const int t = (int)threadIdx.x - rot;
  return (t < 0 ? t + (int)blockDim.x : t) * gridDim.x + blockIdx.x;
}
// The same for groups of T consecutive threads (T divides the block size and
// `rot`).
template <int T>
__device__ __forceinline__ int spread_group(int rot = 0) {
  const int t = (int)threadIdx.x - rot;
  return ((t < 0 ? t + (int)blockDim.x : t) / T) * gridDim.x + blockIdx.x;
}
// Rotations used by the phases: hub chunks from warp 0, tile items from the
// first warp of the second quarter of the block, one-thread items from the
// middle.
__device__ __forceinline__ int rot_tiles() { return (int)blockDim.x / 4; }
__device__ __forceinline__ int rot_threads() { return (int)blockDim.x / 2; }

// ---- queue append (warp-aggregated) -----------------------------------------
__device__ __forceinline__ void append(int *q, int *tail, int v) {
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(tail, (int)g.size());
  base = g.shfl(base, 0);
  q[base + g.thread_rank()] = v;
}

// append() into a queue of `cap` entries: *tail still counts every append, so
// *tail > cap afterwards tells that entries were dropped.
__device__ __forceinline__ void append_bounded(int *q, int *tail, int v, int cap) {
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(tail, (int)g.size());
  base = g.shfl(base, 0);
  if (base + (int)g.thread_rank() < cap) q[base + g.thread_rank()] = v;
}

__device__ __forceinline__ void agg_add_ll(long long *p, long long v) {
  cg::coalesced_group g = cg::coalesced_threads();
  long long s = cg::reduce(g, v, cg::plus<long long>());
  if (g.thread_rank() == 0 && s) atomic_add_ll(p, s);
}

__device__ __forceinline__ void agg_add_int(int *p, int v) {
  cg::coalesced_group g = cg::coalesced_threads();
  int s = cg::reduce(g, v, cg::plus<int>());
  if (g.thread_rank() == 0 && s) atomicAdd(p, s);
}

// Block-wide sum added with one global atomic: for counters that every warp of
// the grid contributes to at the end of a phase (thousands of same-address
// atomics otherwise serialise at one L2 slice).  Every thread of the block must
// call it (uniform control flow: it contains block barriers).
__device__ __forceinline__ void block_add_ll(long long *p, long long v) {
  __shared__ long long s_acc;
  if (threadIdx.x == 0) s_acc = 0;
  __syncthreads();
  cg::thread_block_tile<32> w = cg::tiled_partition<32>(cg::this_thread_block());
  const long long sw = cg::reduce(w, v, cg::plus<long long>());
  if (w.thread_rank() == 0 && sw) atomicAdd((unsigned long long *)&s_acc, (unsigned long long)sw);
  __syncthreads();
  if (threadIdx.x == 0 && s_acc) atomic_add_ll(p, s_acc);
  __syncthreads();
}

__device__ __forceinline__ void block_add_int(int *p, int v) {
  __shared__ int s_acc;
  if (threadIdx.x == 0) s_acc = 0;
  __syncthreads();
  cg::thread_block_tile<32> w = cg::tiled_partition<32>(cg::this_thread_block());
  const int sw = cg::reduce(w, v, cg::plus<int>());
  if (w.thread_rank() == 0 && sw) atomicAdd(&s_acc, sw);
  __syncthreads();
  if (threadIdx.x == 0 && s_acc) atomicAdd(p, s_acc);
  __syncthreads();
}

// ---- groups: one thread, T lanes of a warp, or the whole block ----------------
struct ThreadGroup {
  __device__ __forceinline__ int rank() const { return 0; }
  __host__ __device__ static constexpr int size() { return 1; }
  __device__ __forceinline__ long long scan(long long x, long long &tot) {
    tot = x;
    return 0;
  }
  __device__ __forceinline__ int min_all(int x) { return x; }
  __device__ __forceinline__ long long sum_all(long long x) { return x; }
  __device__ __forceinline__ bool any(bool x) { return x; }
};

template <int T>
struct TileGroup {
  cg::thread_block_tile<T> g;
  __device__ TileGroup() : g(cg::tiled_partition<T>(cg::this_thread_block())) {}
  __device__ __forceinline__ int rank() const { return (int)g.thread_rank(); }
  __host__ __device__ static constexpr int size() { return T; }
  // exclusive prefix sum and total
  __device__ __forceinline__ long long scan(long long x, long long &tot) {
    long long pre = cg::exclusive_scan(g, x, cg::plus<long long>());
    tot = g.shfl(pre + x, T - 1);
    return pre;
  }
  __device__ __forceinline__ int min_all(int x) { return cg::reduce(g, x, cg::less<int>()); }
  __device__ __forceinline__ long long sum_all(long long x) { return cg::reduce(g, x, cg::plus<long long>()); }
  __device__ __forceinline__ bool any(bool x) { return g.any(x); }
};

template <int BLOCK>
struct BlockGroup {
  typedef cub::BlockScan<long long, BLOCK> Scan;
  typedef cub::BlockReduce<int, BLOCK> RedI;
  typedef cub::BlockReduce<long long, BLOCK> RedL;
  union Temp {
    typename Scan::TempStorage scan;
    typename RedI::TempStorage redi;
    typename RedL::TempStorage redl;
  };
  Temp &tmp;
  int *bcast_i;
  long long *bcast_l;
  __device__ BlockGroup(Temp &t, int *bi, long long *bl) : tmp(t), bcast_i(bi), bcast_l(bl) {}
  __device__ __forceinline__ int rank() const { return (int)threadIdx.x; }
  __host__ __device__ static constexpr int size() { return BLOCK; }
  __device__ __forceinline__ long long scan(long long x, long long &tot) {
    long long pre;
    __syncthreads();
    Scan(tmp.scan).ExclusiveSum(x, pre, tot);
    return pre;
  }
  __device__ __forceinline__ int min_all(int x) {
    __syncthreads();
    int r = RedI(tmp.redi).Reduce(x, cub::Min());
    if (threadIdx.x == 0) *bcast_i = r;
    __syncthreads();
    return *bcast_i;
  }
  __device__ __forceinline__ long long sum_all(long long x) {
    __syncthreads();
    long long r = RedL(tmp.redl).Sum(x);
    if (threadIdx.x == 0) *bcast_l = r;
    __syncthreads();
    return *bcast_l;
  }
};


// ---- arc table: (tail, head) -> arc ------------------------------------------
// Open addressing with linear probing over `nslots` 16-byte slots.  An empty
// slot has tail == kEmptyTail (the table is cleared with 0xFF bytes, which also
// sets arc = -1).  The table is only read after it is built: a lookup does not
// write the slot line, so the line is never written back.
struct __align__(16) ArcSlot {
  int tail, head, arc, unused;
};
constexpr int kEmptyTail = -1;

// Slots per arc count: load factor at most 0.5, so a found key takes 1.5
// probes on average, most of them in the first slot's DRAM sector (at R-MAT
// 24 the lookup phase measured 291 us at load 0.5, 340 us at 0.62, 540 us at
// 0.8, for 2.6 M updates).
__host__ __device__ constexpr long long arc_table_slots(long long m) { return 2 * m + 64; }

// The 64-bit key as it lies in the slot's first two words (tail low, head high).
__device__ __forceinline__ unsigned long long arc_key(int u, int v) {
  return ((unsigned long long)(unsigned)v << 32) | (unsigned)u;
}

// First slot of a key: the SplitMix64 finaliser (Steele, Lea and Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014) mixes the
// key, and the high half of its product with nslots maps it onto [0, nslots)
// (Lemire's multiply-shift range reduction) without a division.
__device__ __forceinline__ long long arc_slot0(int u, int v, long long nslots) {
  unsigned long long x = arc_key(u, v);
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return (long long)__umul64hi(x, (unsigned long long)nslots);
}

// One slot as one 16-byte load through L2, bypassing L1: a random slot is
// seldom read twice by one SM, and tail, head and arc never change after the
// build.
__device__ __forceinline__ ArcSlot load_slot(const ArcSlot *s) {
  const int4 x = __ldcg(reinterpret_cast<const int4 *>(s));
  return ArcSlot{x.x, x.y, x.z, x.w};
}

// Arc u->v, or -1 (read-only probe).
__device__ __forceinline__ int find_arc_table(const ArcSlot *tab, long long nslots, int u, int v) {
  long long sl = arc_slot0(u, v, nslots);
  for (long long probe = 0; probe < nslots; probe++) {
    const ArcSlot s = load_slot(tab + sl);
    if (s.tail == u && s.head == v) return s.arc;
    if (s.tail == kEmptyTail) return -1;
    sl = sl + 1 == nslots ? 0 : sl + 1;
  }
  return -1;
}

}  // namespace dmfd
