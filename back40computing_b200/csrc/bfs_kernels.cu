// sm_100a BFS kernels: expand-contract, contract-expand and two-phase.
//
// Each strategy exists as (a) one persistent cooperative kernel that runs every
// BFS level and synchronises levels with the bounded grid barrier (the
// reference's KernelGlobalBarrier, contract_expand_atomic/kernel.cuh:281-554,
// expand_contract_atomic/kernel.cuh:691, two_phase/kernel.cuh:60-313), and
// (b) per-level kernels driven by a CUDA graph with a conditional-while node
// (the reference's EnactIterativeSearch host loops, enactor_contract_expand.cuh:
// 416-516, enactor_two_phase.cuh:465-598), which keeps the level loop on the
// device instead of polling a host-mapped "done" word.
//
// Neighbour-list gather follows the reference's three-way split by list length
// (two_phase/expand_atomic/cta.cuh:215-423): lists >= cta_th are streamed by the
// whole CTA, lists >= warp_th by one warp, and shorter lists are packed into a
// shared-memory gather-offset scratch by a block-wide prefix sum and read by the
// CTA together.  Two additions: CTA and warp lists are read with 16-byte
// vector loads that carry an L2 evict_first policy, and lists >= big_th are
// deferred to a grid-wide phase in which every CTA takes chunks of them, so one
// hub vertex cannot serialise a level behind a single CTA.
//
// Culling: the visited bitmask is the authority and is updated with atomicOr
// (exact), so each vertex is labelled and expanded once; optional warp-level
// (__match_any_sync) and per-CTA history-hash culls drop repeats before they
// reach the mask (contract_atomic/cta.cuh:276-327).

#include <cuda_runtime.h>

#include <cstddef>

#include "bfs_kernels.cuh"

namespace b40c_b200 {

constexpr unsigned FULL = 0xffffffffu;
constexpr int HIST_SIZE = 1024;  // history-hash entries per CTA
constexpr unsigned NO_SPACE = 0xffffffffu;

template <int THREADS, bool MP>
struct Smem {
    static constexpr int SCRATCH = THREADS * 4;  // gather-offset scratch entries
    int2 warp_tot[THREADS / 32 + 1];
    int gofs[SCRATCH];
    int gpred[MP ? SCRATCH : 1];
    int hist[HIST_SIZE];
    int owner;
    int c_start, c_len, c_pred;
    unsigned c_out;
    unsigned tile;
    unsigned out_base;
    unsigned flag;
};

// ---------------------------------------------------------------------------------------
// Sinks: what happens to each gathered neighbour.  Called by every lane of a
// warp together (valid marks the lanes that hold an element).
// ---------------------------------------------------------------------------------------

// Optional culls shared by both kinds of sink.  Returns the surviving validity.
template <int THREADS, bool MP>
__device__ __forceinline__ bool pre_cull(bool valid, int u, unsigned flags, Smem<THREADS, MP> &sm) {
    if (flags & CULL_WARP) {
        // Lanes without an element get distinct negative keys so they never match.
        int key = valid ? u : int(0x80000000u | lane_id());
        unsigned peers = __match_any_sync(FULL, key);
        if (valid && (int)lane_id() != __ffs(peers) - 1) valid = false;
    }
    if ((flags & CULL_HISTORY) && valid) {
        int h = u & (HIST_SIZE - 1);
        if (sm.hist[h] == u) valid = false;  // seen recently by this CTA
        else sm.hist[h] = u;                 // racy insert is harmless
    }
    return valid;
}

// Expand-contract: mark and label each neighbour, then enqueue the ones this
// thread discovered with one atomicAdd per warp.
template <int THREADS, bool MP>
struct DiscoverSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int *q_out;
    unsigned *qlen_out;
    int label;  // iteration + 1

    __device__ __forceinline__ void operator()(bool valid, int u, int pred, unsigned) const {
        bool disc = false;
        valid = pre_cull<THREADS, MP>(valid, u, p.cull_flags, sm);
        if (valid) {
            if ((unsigned)u >= (unsigned)p.nodes) {
                atomicOr(&p.ctr->error, ERR_BAD_VERTEX);
            } else if (mark_visited(p.mask, u)) {
                disc = true;
                p.labels[u] = MP ? pred : label;
            }
        }
        unsigned b = __ballot_sync(FULL, disc);
        if (b) {
            int leader = __ffs(b) - 1;
            unsigned base = 0;
            if ((int)lane_id() == leader) base = atomicAdd(qlen_out, (unsigned)__popc(b));
            base = __shfl_sync(FULL, base, leader);
            if (disc) {
                unsigned long long pos = (unsigned long long)base + __popc(b & lanemask_lt());
                if (pos < (unsigned long long)p.qcap) q_out[pos] = u;
                else atomicOr(&p.ctr->error, ERR_OVERFLOW);
            }
        }
    }
};

// Contract-expand / two-phase expand: neighbours are written at positions
// reserved beforehand by a block-wide scan (edge frontier, duplicates kept).
template <bool MP>
struct PositionSink {
    int *q_out;
    int *pq_out;
    __device__ __forceinline__ void operator()(bool valid, int u, int pred, unsigned pos) const {
        if (valid) {
            q_out[pos] = u;
            if (MP) pq_out[pos] = pred;
        }
    }
};

// ---------------------------------------------------------------------------------------
// Gather strategies
// ---------------------------------------------------------------------------------------

// The calling group (CTA of THREADS, or one warp with GROUP = 32) streams list
// [s, s+l) with 16-byte loads from the aligned-down start; elements outside the
// list are masked off.  col must have 3 readable entries past the last edge.
template <int GROUP, class Sink>
__device__ __forceinline__ void gather_list(const int *col, int vec_end, int s, int l, int pred,
                                            unsigned out, int rank, const Sink &sink, uint64_t pol) {
    const int end = s + l;
    for (int base = s & ~3; base < end; base += GROUP * 4) {
        int e = base + rank * 4;
        int4 c = make_int4(-1, -1, -1, -1);
        if (e < end) {
            if (e + 4 <= vec_end) {
                c = ldg_stream_v4(col + e, pol);
            } else {  // unpadded (host-mapped) array tail: scalar loads inside the list
                c.x = __ldg(col + e);
                if (e + 1 < end) c.y = __ldg(col + e + 1);
                if (e + 2 < end) c.z = __ldg(col + e + 2);
                if (e + 3 < end) c.w = __ldg(col + e + 3);
            }
        }
        sink(e >= s && e < end, c.x, pred, out + unsigned(e - s));
        sink(e + 1 >= s && e + 1 < end, c.y, pred, out + unsigned(e + 1 - s));
        sink(e + 2 >= s && e + 2 < end, c.z, pred, out + unsigned(e + 2 - s));
        sink(e + 3 >= s && e + 3 < end, c.w, pred, out + unsigned(e + 3 - s));
    }
}

// CTA-, warp- and scan-based gather of the lists held by the CTA's threads
// (one list per thread: start, len, owner vertex pred, output position out).
// small_off / small_total: block exclusive scan of the lengths of lists shorter
// than warp_th, whose outputs are contiguous from small_base.
template <int THREADS, bool MP, class Sink>
__device__ __forceinline__ void expand_lists(const BfsParams &p, Smem<THREADS, MP> &sm,
                                             const Sink &sink, uint64_t pol, int start, int len,
                                             int pred, unsigned out, int small_off,
                                             int small_total, unsigned small_base) {
    const bool small = len < p.warp_th;
    // (1) whole-CTA gather of lists >= cta_th, one list at a time
    for (;;) {
        if (threadIdx.x == 0) sm.owner = -1;
        __syncthreads();
        if (len >= p.cta_th) sm.owner = threadIdx.x;
        __syncthreads();
        int owner = sm.owner;
        if (owner < 0) break;
        if (owner == (int)threadIdx.x) {
            sm.c_start = start;
            sm.c_len = len;
            sm.c_pred = pred;
            sm.c_out = out;
            len = 0;
        }
        __syncthreads();
        gather_list<THREADS>(p.col, p.vec_end, sm.c_start, sm.c_len, sm.c_pred, sm.c_out, threadIdx.x, sink, pol);
    }
    // (2) warp gather of lists >= warp_th
    unsigned wm;
    while ((wm = __ballot_sync(FULL, len >= p.warp_th)) != 0u) {
        int leader = __ffs(wm) - 1;
        int s = __shfl_sync(FULL, start, leader);
        int l = __shfl_sync(FULL, len, leader);
        int pv = __shfl_sync(FULL, pred, leader);
        unsigned o = __shfl_sync(FULL, out, leader);
        if ((int)lane_id() == leader) len = 0;
        gather_list<32>(p.col, p.vec_end, s, l, pv, o, lane_id(), sink, pol);
    }
    // (3) scan-based gather of the short lists through shared memory
    constexpr int SCRATCH = Smem<THREADS, MP>::SCRATCH;
    const int my_len = small ? len : 0;
    for (int round = 0; round < small_total; round += SCRATCH) {
        int lo = max(small_off, round), hi = min(small_off + my_len, round + SCRATCH);
        for (int j = lo; j < hi; j++) {
            sm.gofs[j - round] = start + (j - small_off);
            if (MP) sm.gpred[j - round] = pred;
        }
        __syncthreads();
        const int cnt = min(SCRATCH, small_total - round);
        for (int k0 = 0; k0 < cnt; k0 += THREADS) {
            int k = k0 + threadIdx.x;
            bool valid = k < cnt;
            int u = -1, pv = 0;
            if (valid) {
                u = __ldg(p.col + sm.gofs[k]);
                if (MP) pv = sm.gpred[k];
            }
            sink(valid, u, pv, small_base + unsigned(round + k));
        }
        __syncthreads();
    }
}

// Grid-wide phase: every CTA takes chunks of the deferred big lists, chunk g of
// the concatenated chunk sequence going to CTA g mod gridDim.x.
template <int THREADS, class Sink>
__device__ __forceinline__ void gather_big_lists(const BfsParams &p, unsigned nbig, const Sink &sink,
                                                 uint64_t pol) {
    constexpr int CHUNK = THREADS * 16;
    const unsigned G = gridDim.x;
    unsigned g0 = 0;
    if (nbig > (unsigned)p.big_cap) nbig = p.big_cap;
    for (unsigned i = 0; i < nbig; i++) {
        int4 item = __ldcg(p.big_items + i);
        int s = item.x, l = item.y;
        unsigned chunks = unsigned((l + CHUNK - 1) / CHUNK);
        unsigned c = (blockIdx.x + G - (g0 % G)) % G;
        for (; c < chunks; c += G) {
            int cs = s + int(c) * CHUNK;
            int cl = min(CHUNK, l - int(c) * CHUNK);
            gather_list<THREADS>(p.col, p.vec_end, cs, cl, item.z, unsigned(item.w) + c * CHUNK, threadIdx.x, sink,
                                 pol);
        }
        g0 += chunks;
    }
}

// Hand out tiles of the input frontier to CTAs with one atomic each.
template <int THREADS, bool MP>
__device__ __forceinline__ unsigned next_tile(unsigned *steal, Smem<THREADS, MP> &sm) {
    __syncthreads();
    if (threadIdx.x == 0) sm.tile = atomicAdd(steal, 1u);
    __syncthreads();
    return sm.tile;
}

// Defers a list to the grid-wide phase; returns true when it was taken.
__device__ __forceinline__ bool push_big(const BfsParams &p, unsigned *bigc, int start, int len,
                                         int pred, unsigned out) {
    unsigned item = atomicAdd(bigc, 1u);
    if (item < (unsigned)p.big_cap) {
        p.big_items[item] = make_int4(start, len, pred, int(out));
        return true;
    }
    return false;  // table full: the caller's CTA gathers the list itself
}

__device__ __forceinline__ void row_range(const BfsParams &p, int v, int &start, int &len) {
    start = __ldg(p.row_offsets + v);
    len = __ldg(p.row_offsets + v + 1) - start;
}

// ---------------------------------------------------------------------------------------
// Level bodies
// ---------------------------------------------------------------------------------------

// Expand-contract level `it`: vertex frontier queue[it&1] -> queue[(it+1)&1].
// Neighbours are labelled it+1 when discovered (expand_contract_atomic/cta.cuh:
// 181-218).  Lists >= big_th are deferred to big[it&3].
template <int THREADS, bool MP>
__device__ void ec_level(const BfsParams &p, int it, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[it & 1];
    DiscoverSink<THREADS, MP> sink{p, sm, p.queue[(it + 1) & 1], &c->qlen[(it + 1) & 3], it + 1};
    const unsigned ntiles = (L + THREADS - 1) / THREADS;
    for (;;) {
        unsigned tile = next_tile<THREADS, MP>(&c->steal[it & 3], sm);
        if (tile >= ntiles) break;
        unsigned idx = tile * THREADS + threadIdx.x;
        int v = -1, start = 0, len = 0;
        if (idx < L) {
            v = ld_cg(q_in + idx);
            row_range(p, v, start, len);
            if (len >= p.big_th && push_big(p, &c->big[it & 3], start, len, v, 0u)) len = 0;
        }
        int small_total;
        int small_off = block_exclusive_scan<THREADS>(len < p.warp_th ? len : 0, small_total, sm.warp_tot);
        expand_lists<THREADS, MP>(p, sm, sink, pol, start, len, v, 0u, small_off, small_total, 0u);
    }
}

template <int THREADS, bool MP>
__device__ void ec_big(const BfsParams &p, int it, unsigned nbig, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    DiscoverSink<THREADS, MP> sink{p, sm, p.queue[(it + 1) & 1], &c->qlen[(it + 1) & 3], it + 1};
    gather_big_lists<THREADS>(p, nbig, sink, pol);
}

// Expands the per-thread lists (start, len, owner pred) of one tile into the
// edge frontier queue q_out: a two-component block scan sizes the short and
// the long lists, thread 0 reserves the tile's output with one atomicAdd
// (ScanTileWithEnqueue, util/scan/cooperative_scan.cuh:173-195), big lists are
// deferred with their reserved output position.
template <int THREADS, bool MP>
__device__ __forceinline__ void expand_tile_to_edges(const BfsParams &p, Smem<THREADS, MP> &sm,
                                                     uint64_t pol, int start, int len, int pred,
                                                     int *q_out, int *pq_out, unsigned *qlen_out,
                                                     unsigned *bigc) {
    const bool small = len < p.warp_th;
    int2 total;
    int2 off = block_exclusive_scan2<THREADS>(make_int2(small ? len : 0, small ? 0 : len), total,
                                              sm.warp_tot);
    if (threadIdx.x == 0) {
        unsigned need = unsigned(total.x + total.y);
        unsigned base = 0;
        if (need) {
            base = atomicAdd(qlen_out, need);
            if ((unsigned long long)base + need > (unsigned long long)p.qcap) {
                atomicOr(&p.ctr->error, ERR_OVERFLOW);
                base = NO_SPACE;
            }
        }
        sm.out_base = base;
    }
    __syncthreads();
    const unsigned base = sm.out_base;
    if (base == NO_SPACE) return;  // uniform: the whole tile is dropped on overflow
    const unsigned small_base = base;
    unsigned out = small ? small_base + off.x : base + unsigned(total.x) + off.y;
    if (len >= p.big_th && push_big(p, bigc, start, len, pred, out)) len = 0;
    PositionSink<MP> sink{q_out, pq_out};
    expand_lists<THREADS, MP>(p, sm, sink, pol, start, len, pred, out, off.x, total.x, small_base);
}

// Culls one edge-frontier element: optional warp / history culls, then the
// exact bitmask test-and-set.  Survivors are labelled (iteration or pred).
template <int THREADS, bool MP>
__device__ __forceinline__ bool contract_one(const BfsParams &p, Smem<THREADS, MP> &sm, bool valid,
                                             int u, int pred, int it) {
    valid = pre_cull<THREADS, MP>(valid, u, p.cull_flags, sm);
    if (valid) {
        if ((unsigned)u >= (unsigned)p.nodes) {
            atomicOr(&p.ctr->error, ERR_BAD_VERTEX);
            valid = false;
        } else if (mark_visited(p.mask, u)) {
            p.labels[u] = MP ? pred : it;
        } else {
            valid = false;
        }
    }
    return valid;
}

// Contract-expand level `it` (contract_expand_atomic/cta.cuh:573-709): edge
// frontier queue[it&1] -> cull + label it -> expand -> queue[(it+1)&1].
template <int THREADS, bool MP>
__device__ void ce_level(const BfsParams &p, int it, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[it & 1];
    const int *pq_in = p.pred_queue[it & 1];
    const unsigned ntiles = (L + THREADS - 1) / THREADS;
    for (;;) {
        unsigned tile = next_tile<THREADS, MP>(&c->steal[it & 3], sm);
        if (tile >= ntiles) break;
        unsigned idx = tile * THREADS + threadIdx.x;
        bool valid = idx < L;
        int u = -1, pred = 0;
        if (valid) {
            u = ld_cg(q_in + idx);
            if (MP) pred = ld_cg(pq_in + idx);
        }
        valid = contract_one<THREADS, MP>(p, sm, valid, u, pred, it);
        int start = 0, len = 0;
        if (valid) row_range(p, u, start, len);
        expand_tile_to_edges<THREADS, MP>(p, sm, pol, start, len, u, p.queue[(it + 1) & 1],
                                          p.pred_queue[(it + 1) & 1], &c->qlen[(it + 1) & 3],
                                          &c->big[it & 3]);
    }
}

template <int THREADS, bool MP>
__device__ void edges_big(const BfsParams &p, int out_sel, unsigned nbig, uint64_t pol) {
    PositionSink<MP> sink{p.queue[out_sel], p.pred_queue[out_sel]};
    gather_big_lists<THREADS>(p, nbig, sink, pol);
}

// Two-phase contract (two_phase/contract_atomic/cta.cuh:494-572): edge frontier
// queue[qi&1] -> cull + label `it` -> compacted vertex frontier queue[(qi+1)&1],
// allocated by a block scan and one atomicAdd per tile.
template <int THREADS, bool MP>
__device__ void tp_contract(const BfsParams &p, int it, int qi, unsigned L, Smem<THREADS, MP> &sm) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[qi & 1];
    const int *pq_in = p.pred_queue[qi & 1];
    int *q_out = p.queue[(qi + 1) & 1];
    const unsigned ntiles = (L + THREADS - 1) / THREADS;
    for (;;) {
        unsigned tile = next_tile<THREADS, MP>(&c->steal[qi & 3], sm);
        if (tile >= ntiles) break;
        unsigned idx = tile * THREADS + threadIdx.x;
        bool valid = idx < L;
        int u = -1, pred = 0;
        if (valid) {
            u = ld_cg(q_in + idx);
            if (MP) pred = ld_cg(pq_in + idx);
        }
        valid = contract_one<THREADS, MP>(p, sm, valid, u, pred, it);
        int total;
        int off = block_exclusive_scan<THREADS>(valid ? 1 : 0, total, sm.warp_tot);
        if (threadIdx.x == 0) {
            unsigned base = total ? atomicAdd(&c->qlen[(qi + 1) & 3], (unsigned)total) : 0u;
            if ((unsigned long long)base + total > (unsigned long long)p.qcap) {
                atomicOr(&c->error, ERR_OVERFLOW);
                base = NO_SPACE;
            }
            sm.out_base = base;
        }
        __syncthreads();
        if (valid && sm.out_base != NO_SPACE) q_out[sm.out_base + off] = u;
    }
}

// Two-phase expand (two_phase/expand_atomic/cta.cuh:606-719): vertex frontier
// queue[qi&1] -> edge frontier queue[(qi+1)&1] with predecessors.
template <int THREADS, bool MP>
__device__ void tp_expand(const BfsParams &p, int qi, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[qi & 1];
    const unsigned ntiles = (L + THREADS - 1) / THREADS;
    for (;;) {
        unsigned tile = next_tile<THREADS, MP>(&c->steal[qi & 3], sm);
        if (tile >= ntiles) break;
        unsigned idx = tile * THREADS + threadIdx.x;
        int v = -1, start = 0, len = 0;
        if (idx < L) {
            v = ld_cg(q_in + idx);
            row_range(p, v, start, len);
        }
        expand_tile_to_edges<THREADS, MP>(p, sm, pol, start, len, v, p.queue[(qi + 1) & 1],
                                          p.pred_queue[(qi + 1) & 1], &c->qlen[(qi + 1) & 3],
                                          &c->big[qi & 3]);
    }
}

// Ring housekeeping for phase index q: entries that phase q+1 will use start
// from zero.  Done by one thread while no CTA touches them.
__device__ __forceinline__ void ring_prepare(Counters *c, int q) {
    c->qlen[(q + 2) & 3] = 0u;
    c->steal[(q + 1) & 3] = 0u;
    c->big[(q + 1) & 3] = 0u;
}

template <int THREADS, bool MP>
__device__ __forceinline__ void init_hist(Smem<THREADS, MP> &sm, unsigned flags) {
    if (flags & CULL_HISTORY)
        for (int i = threadIdx.x; i < HIST_SIZE; i += THREADS) sm.hist[i] = -1;
}

// ---------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------

// Per-search initialisation: counters and barrier to zero, the source in the
// first frontier.  Expand-contract labels and marks the source here (as
// expand_contract_atomic/kernel.cuh:291-326); the edge-frontier strategies
// label it when they contract it at iteration 0, with predecessor -2.
__global__ void search_init_kernel(BfsParams p, int strategy, int mark_pred) {
    Counters *c = p.ctr;
    unsigned *w = reinterpret_cast<unsigned *>(c);
    constexpr int WORDS = int(offsetof(Counters, sticky) / 4);  // everything but the sticky error
    for (int i = threadIdx.x; i < WORDS; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        c->qlen[0] = 1u;
        p.queue[0][0] = p.src;
        if (strategy == STRATEGY_EXPAND_CONTRACT) {
            p.labels[p.src] = mark_pred ? -2 : 0;
            p.mask[unsigned(p.src) >> 5] |= 1u << (unsigned(p.src) & 31u);
        } else if (mark_pred) {
            p.pred_queue[0][0] = -2;
        }
    }
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ec_fused_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int it = 0;
    for (;;) {
        unsigned L = ld_cg(&c->qlen[it & 3]);
        if (L == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ring_prepare(c, it);
            c->total_queued += L;
        }
        ec_level<THREADS, MP>(p, it, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        unsigned nbig = ld_cg(&c->big[it & 3]);
        if (nbig) {
            ec_big<THREADS, MP>(p, it, nbig, sm, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        it++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->iteration = it;
        atomicOr(&c->sticky, ld_relaxed_gpu(&c->error));
    }
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ce_fused_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int it = 0;
    for (;;) {
        unsigned L = ld_cg(&c->qlen[it & 3]);
        if (L == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ring_prepare(c, it);
            c->total_queued += L;
        }
        ce_level<THREADS, MP>(p, it, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        unsigned nbig = ld_cg(&c->big[it & 3]);
        if (nbig) {
            edges_big<THREADS, MP>(p, (it + 1) & 1, nbig, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        it++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->iteration = it;
        atomicOr(&c->sticky, ld_relaxed_gpu(&c->error));
    }
}

// Fused two-phase: contract and expand phases alternate across grid barriers
// (the reference's fused two-phase kernel, two_phase/kernel.cuh:60-313, which
// its enactor cannot instantiate, enactor_two_phase.cuh:302).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_fused_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int it = 0, qi = 0;
    for (;;) {
        unsigned L = ld_cg(&c->qlen[qi & 3]);
        if (L == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ring_prepare(c, qi);
            c->total_queued += L;
        }
        tp_contract<THREADS, MP>(p, it, qi, L, sm);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        qi++;
        L = ld_cg(&c->qlen[qi & 3]);
        if (L == 0u) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) ring_prepare(c, qi);
        tp_expand<THREADS, MP>(p, qi, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        unsigned nbig = ld_cg(&c->big[qi & 3]);
        if (nbig) {
            edges_big<THREADS, MP>(p, (qi + 1) & 1, nbig, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        qi++;
        it++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->iteration = it;
        atomicOr(&c->sticky, ld_relaxed_gpu(&c->error));
    }
}

// ---- per-level kernels for the graph-driven (iterative) variants ----------------

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ec_level_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = *(volatile int *)&p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3];
    if (L == 0u || p.ctr->error) return;
    ec_level<THREADS, MP>(p, it, L, sm, policy_evict_first());
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ec_big_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned nbig = p.ctr->big[it & 3];
    if (nbig == 0u || p.ctr->error) return;
    ec_big<THREADS, MP>(p, it, nbig, sm, policy_evict_first());
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ce_level_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3];
    if (L == 0u || p.ctr->error) return;
    ce_level<THREADS, MP>(p, it, L, sm, policy_evict_first());
}

// Grid-wide big-list pass after a level that writes an edge frontier; `phase`
// is the ring index of that level (iteration for contract-expand, qi+1 for the
// two-phase expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) edges_big_kernel(BfsParams p, int two_phase) {
    const int q = two_phase ? p.ctr->cur_it * 2 + 1 : p.ctr->cur_it;
    const unsigned nbig = p.ctr->big[q & 3];
    if (nbig == 0u || p.ctr->error) return;
    edges_big<THREADS, MP>(p, (q + 1) & 1, nbig, policy_evict_first());
}

// Two-phase per-level: qi = 2 * it (contract) and 2 * it + 1 (expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_contract_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it;
    const unsigned L = p.ctr->qlen[qi & 3];
    if (L == 0u || p.ctr->error) return;
    tp_contract<THREADS, MP>(p, it, qi, L, sm);
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_expand_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it + 1;
    const unsigned L = p.ctr->qlen[qi & 3];
    if (L == 0u || p.ctr->error) return;
    tp_expand<THREADS, MP>(p, qi, L, sm, policy_evict_first());
}

// Runs alone between levels of a per-level graph: records the level, prepares
// the ring for the next one and sets the while-loop condition.
__global__ void level_control_kernel(BfsParams p, int strategy) {
    if (threadIdx.x != 0) return;
    Counters *c = p.ctr;
    const int it = c->cur_it;
    bool more;
    if (strategy == STRATEGY_TWO_PHASE) {
        const int qi = 2 * it;
        const unsigned vq = c->qlen[(qi + 1) & 3];  // contract output
        const unsigned eq = c->qlen[(qi + 2) & 3];  // expand output
        c->total_queued += c->qlen[qi & 3];
        if (vq == 0u) {
            c->iteration = it;  // reference breaks after contract without ++
            more = false;
        } else {
            c->iteration = it + 1;
            more = eq != 0u;
        }
        // next body runs phases qi+2 (contract) and qi+3 (expand)
        c->steal[(qi + 2) & 3] = 0u;
        c->steal[(qi + 3) & 3] = 0u;
        c->qlen[(qi + 3) & 3] = 0u;
        c->qlen[(qi + 4) & 3] = 0u;
        c->big[(qi + 3) & 3] = 0u;
    } else {
        const unsigned next = c->qlen[(it + 1) & 3];
        c->total_queued += c->qlen[it & 3];
        c->iteration = it + 1;
        more = next != 0u;
        c->steal[(it + 1) & 3] = 0u;
        c->big[(it + 1) & 3] = 0u;
        c->qlen[(it + 2) & 3] = 0u;
    }
    if (more && level_limit_hit(it + 1, p.nodes)) {
        c->error |= ERR_LEVEL_LIMIT;
        more = false;
    }
    if (c->error) more = false;
    c->cur_it = it + 1;
    if (!more) {
        c->done = 1u;
        c->sticky |= c->error;
    }
    cudaGraphSetConditional((cudaGraphConditionalHandle)p.cond_handle, more ? 1u : 0u);
}

// Failure-detection probe: the barrier waits for gridDim.x + 1 arrivals, so no
// CTA is ever released and each one leaves after wait_ns.
__global__ void barrier_timeout_probe_kernel(Counters *c, unsigned long long wait_ns) {
    __shared__ unsigned flag;
    grid_barrier(c, wait_ns, &flag, gridDim.x + 1u);
}

// ---------------------------------------------------------------------------------------
// Host-side dispatch
// ---------------------------------------------------------------------------------------

typedef void (*KernelFn)(BfsParams);

template <int THREADS, bool MP>
static KernelFn fused_fn(int strategy) {
    switch (strategy) {
    case STRATEGY_EXPAND_CONTRACT: return ec_fused_kernel<THREADS, MP>;
    case STRATEGY_CONTRACT_EXPAND: return ce_fused_kernel<THREADS, MP>;
    default: return tp_fused_kernel<THREADS, MP>;
    }
}

template <bool MP>
static KernelFn fused_fn_t(int threads, int strategy) {
    switch (threads) {
    case 128: return fused_fn<128, MP>(strategy);
    case 512: return fused_fn<512, MP>(strategy);
    default: return fused_fn<256, MP>(strategy);
    }
}

static KernelFn pick_fused(const KernelConfig &kc) {
    return kc.mark_pred ? fused_fn_t<true>(kc.threads, kc.strategy)
                        : fused_fn_t<false>(kc.threads, kc.strategy);
}

struct LevelFns {
    KernelFn level_a;  // ec_level / ce_level / tp_contract
    KernelFn level_b;  // ec_big / (none) / tp_expand
    void (*edges_big)(BfsParams, int);
};

template <int THREADS, bool MP>
static LevelFns level_fns(int strategy) {
    LevelFns f{};
    f.edges_big = edges_big_kernel<THREADS, MP>;
    switch (strategy) {
    case STRATEGY_EXPAND_CONTRACT:
        f.level_a = ec_level_kernel<THREADS, MP>;
        f.level_b = ec_big_kernel<THREADS, MP>;
        break;
    case STRATEGY_CONTRACT_EXPAND:
        f.level_a = ce_level_kernel<THREADS, MP>;
        f.level_b = nullptr;
        break;
    default:
        f.level_a = tp_contract_kernel<THREADS, MP>;
        f.level_b = tp_expand_kernel<THREADS, MP>;
        break;
    }
    return f;
}

template <bool MP>
static LevelFns level_fns_t(int threads, int strategy) {
    switch (threads) {
    case 128: return level_fns<128, MP>(strategy);
    case 512: return level_fns<512, MP>(strategy);
    default: return level_fns<256, MP>(strategy);
    }
}

static LevelFns pick_level(const KernelConfig &kc) {
    return kc.mark_pred ? level_fns_t<true>(kc.threads, kc.strategy)
                        : level_fns_t<false>(kc.threads, kc.strategy);
}

static cudaError_t grid_for(const void *fn, int threads, int *grid) {
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, 0);
    if (e) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    *grid = sms * occ;
    return cudaSuccess;
}

cudaError_t launch_search_init(const BfsParams &p, const KernelConfig &kc, cudaStream_t stream) {
    search_init_kernel<<<1, 64, 0, stream>>>(p, kc.strategy, kc.mark_pred ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t fused_grid_limit(const KernelConfig &kc, int *grid) {
    return grid_for((const void *)pick_fused(kc), kc.threads, grid);
}

cudaError_t level_grid_limit(const KernelConfig &kc, int *grid) {
    return grid_for((const void *)pick_level(kc).level_a, kc.threads, grid);
}

cudaError_t launch_fused(const BfsParams &p, const KernelConfig &kc, int grid, cudaStream_t stream) {
    KernelFn fn = pick_fused(kc);
    BfsParams arg = p;
    void *args[] = {&arg};
    return cudaLaunchCooperativeKernel((const void *)fn, dim3(grid), dim3(kc.threads), args, 0, stream);
}

cudaError_t build_level_graph(BfsParams &p, const KernelConfig &kc, int grid, cudaGraphExec_t *exec,
                              cudaGraph_t *graph_out) {
    cudaGraph_t graph = nullptr;
    cudaStream_t cap = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e) return e;
    do {
        cudaGraphConditionalHandle handle;
        if ((e = cudaGraphConditionalHandleCreate(&handle, graph, 1u, cudaGraphCondAssignDefault))) break;
        p.cond_handle = (unsigned long long)handle;

        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = handle;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if ((e = cudaGraphAddNode(&node, graph, nullptr, 0, &np))) break;
        cudaGraph_t body = np.conditional.phGraph_out[0];

        if ((e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking))) break;
        if ((e = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal)))
            break;
        LevelFns f = pick_level(kc);
        const int T = kc.threads;
        f.level_a<<<grid, T, 0, cap>>>(p);
        if (kc.strategy == STRATEGY_EXPAND_CONTRACT) {
            f.level_b<<<grid, T, 0, cap>>>(p);
        } else if (kc.strategy == STRATEGY_CONTRACT_EXPAND) {
            f.edges_big<<<grid, T, 0, cap>>>(p, 0);
        } else {
            f.level_b<<<grid, T, 0, cap>>>(p);
            f.edges_big<<<grid, T, 0, cap>>>(p, 1);
        }
        level_control_kernel<<<1, 32, 0, cap>>>(p, kc.strategy);
        cudaError_t le = cudaGetLastError();
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(cap, &captured);
        if (le) e = le;
        if (e) break;
        e = cudaGraphInstantiate(exec, graph, 0);
    } while (0);
    if (cap) cudaStreamDestroy(cap);
    if (e) {
        cudaGraphDestroy(graph);
        return e;
    }
    *graph_out = graph;
    return cudaSuccess;
}

cudaError_t run_barrier_timeout_probe(int grid, unsigned long long wait_ns, unsigned *error_out) {
    Counters *c = nullptr;
    cudaError_t e = cudaMalloc(&c, sizeof(Counters));
    if (e) return e;
    do {
        if ((e = cudaMemset(c, 0, sizeof(Counters)))) break;
        void *args[] = {&c, &wait_ns};
        if ((e = cudaLaunchCooperativeKernel((const void *)barrier_timeout_probe_kernel, dim3(grid),
                                             dim3(32), args, 0, nullptr)))
            break;
        if ((e = cudaDeviceSynchronize())) break;
        Counters h;
        if ((e = cudaMemcpy(&h, c, sizeof(Counters), cudaMemcpyDeviceToHost))) break;
        *error_out = h.error;
    } while (0);
    cudaFree(c);
    return e;
}

}  // namespace b40c_b200
