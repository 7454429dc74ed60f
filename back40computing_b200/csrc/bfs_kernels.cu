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
// Neighbour-list gather follows the reference's split by list length
// (two_phase/expand_atomic/cta.cuh:215-423): lists >= cta_th are streamed by the
// whole CTA, lists >= warp_th by one warp, and shorter lists are packed into a
// shared-memory gather-offset scratch by a block-wide prefix sum and read by the
// CTA together.  A fourth tier takes lists >= big_th: they are cut into
// fixed-size chunks (one 16-byte load per thread of a CTA) that every CTA of
// the grid takes in turn after the tile phase, so a hub vertex never
// serialises a level behind one CTA.  Tiles shrink when the frontier is small
// so that every CTA gets work.  CTA and warp lists are read with 16-byte loads
// carrying an L2 evict_first policy, one pass ahead of use.
//
// Culling: the visited bitmask is the authority and is updated with atomicOr
// (exact), so each vertex is labelled and expanded once.  Each thread tests 4
// elements at a time: 4 mask loads in flight, then at most 4 atomicOr, then one
// warp-aggregated queue reservation.  Optional warp-level (__match_any_sync)
// and per-CTA history-hash culls drop repeats first (contract_atomic/cta.cuh:
// 276-327).

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
    static constexpr int CTILE = THREADS * 4;    // edge-frontier elements per contract tile
    int2 warp_tot[THREADS / 32 + 1];
    int gofs[SCRATCH];
    int gpred[MP ? SCRATCH : 1];
    int hist[HIST_SIZE];
    int surv[CTILE];
    int owner;
    int c_start, c_len, c_pred;
    unsigned c_out;
    unsigned tile;
    unsigned out_base;
    unsigned flag;
};

// ---------------------------------------------------------------------------------------
// Culling and enqueueing, 4 elements per thread
// ---------------------------------------------------------------------------------------

// Optional culls.  Called by every lane of the warp (match_any needs them all).
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

// Exact test-and-set of the visited bits of up to 4 vertices (bit j of valid
// marks u[j]).  Returns the bits of the vertices this thread claimed first.
template <int THREADS, bool MP>
__device__ __forceinline__ unsigned cull4(const BfsParams &p, Smem<THREADS, MP> &sm, unsigned valid,
                                          const int (&u)[4]) {
    if (p.cull_flags) {
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (!pre_cull<THREADS, MP>((valid >> j) & 1u, u[j], p.cull_flags, sm)) valid &= ~(1u << j);
    }
    unsigned w[4], bit[4], m[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        bool ok = (valid >> j) & 1u;
        if (ok && (unsigned)u[j] >= (unsigned)p.nodes) {
            atomicOr(&p.ctr->error, ERR_BAD_VERTEX);
            valid &= ~(1u << j);
            ok = false;
        }
        w[j] = ok ? (unsigned)u[j] >> 5 : 0u;
        bit[j] = 1u << ((unsigned)u[j] & 31u);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) m[j] = ld_cg(p.mask + w[j]);  // 4 probes in flight
    unsigned need = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (((valid >> j) & 1u) && !(m[j] & bit[j])) need |= 1u << j;
    unsigned old[4];
#pragma unroll
    for (int j = 0; j < 4; j++) old[j] = ((need >> j) & 1u) ? atomicOr(p.mask + w[j], bit[j]) : bit[j];
    unsigned claimed = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (!(old[j] & bit[j])) claimed |= 1u << j;
    return claimed;
}

// Appends the flagged elements of every lane to queue q with one atomicAdd
// per warp.  Called by all lanes together.
__device__ __forceinline__ void enqueue4(unsigned flags, const int (&u)[4], int *q, unsigned *qlen, long long qcap,
                                         unsigned *err) {
    const unsigned lt = lanemask_lt();
    unsigned total = 0, pre[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        unsigned b = __ballot_sync(FULL, (flags >> j) & 1u);
        pre[j] = total + __popc(b & lt);
        total += __popc(b);
    }
    if (total == 0u) return;  // warp-uniform
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(qlen, total);
    base = __shfl_sync(FULL, base, 0);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if ((flags >> j) & 1u) {
            unsigned long long pos = (unsigned long long)base + pre[j];
            if (pos < (unsigned long long)qcap) q[pos] = u[j];
            else atomicOr(err, ERR_OVERFLOW);
        }
    }
}

// ---------------------------------------------------------------------------------------
// Sinks: what happens to each gathered neighbour.  Called by every lane of a
// warp together with up to 4 elements per lane; bit j of valid marks u[j];
// output positions are out0 + j.
// ---------------------------------------------------------------------------------------

// Expand-contract: mark and label each neighbour at discovery (label it+1,
// expand_contract_atomic/cta.cuh:181-218), enqueue the discovered ones.
template <int THREADS, bool MP>
struct DiscoverSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int *q_out;
    unsigned *qlen_out;
    int label;

    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pred)[4],
                                               unsigned) const {
        unsigned disc = cull4<THREADS, MP>(p, sm, valid, u);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((disc >> j) & 1u) p.labels[u[j]] = MP ? pred[j] : label;
        enqueue4(disc, u, q_out, qlen_out, p.qcap, &p.ctr->error);
    }
};

// Contract-expand / two-phase expand: neighbours are written at positions
// reserved beforehand by a block-wide scan (edge frontier, duplicates kept).
template <bool MP>
struct PositionSink {
    int *q_out;
    int *pq_out;
    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pred)[4],
                                               unsigned out0) const {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((valid >> j) & 1u) {
                q_out[out0 + j] = u[j];
                if (MP) pq_out[out0 + j] = pred[j];
            }
        }
    }
};

// ---------------------------------------------------------------------------------------
// Gather strategies
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ int4 load_col4(const int *col, int vec_end, int e, int end, uint64_t pol) {
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
    return c;
}

// The calling group (CTA of THREADS, or one warp with GROUP = 32) streams the
// list [s, s+l) with 16-byte loads starting from the 4-aligned index a0 <= s;
// each pass covers GROUP*4 elements; the next pass's load is issued before the
// current elements are processed.  Elements outside [s, s+l) are masked off.
template <int GROUP, class Sink>
__device__ __forceinline__ void gather_list(const int *col, int vec_end, int a0, int s, int l, int pred,
                                            unsigned out, int rank, const Sink &sink, uint64_t pol) {
    const int end = s + l;
    int e = a0 + rank * 4;
    int4 cur = load_col4(col, vec_end, e, end, pol);
    const int pv[4] = {pred, pred, pred, pred};
    for (int base = a0; base < end; base += GROUP * 4) {
        const int en = e + GROUP * 4;
        int4 nxt = load_col4(col, vec_end, en, end, pol);
        unsigned valid = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (e + j >= s && e + j < end) valid |= 1u << j;
        const int u[4] = {cur.x, cur.y, cur.z, cur.w};
        sink(valid, u, pv, out + unsigned(e - s));
        cur = nxt;
        e = en;
    }
}

// CTA-, warp- and scan-based gather of the lists held by the CTA's threads
// (one list per thread: start, len, owner vertex pred, output position out).
// small_off / small_total: block exclusive scan of the lengths of lists shorter
// than warp_th, whose outputs are contiguous from small_base.
template <int THREADS, bool MP, class Sink>
__device__ __forceinline__ void expand_lists(const BfsParams &p, Smem<THREADS, MP> &sm, const Sink &sink,
                                             uint64_t pol, int start, int len, int pred, unsigned out,
                                             int small_off, int small_total, unsigned small_base) {
    const bool small = len < p.warp_th;
    // (1) whole-CTA gather of lists >= cta_th, one list at a time
    for (;;) {
        if (threadIdx.x == 0) sm.owner = -1;
        __syncthreads();
        if (len >= p.cta_th) sm.owner = threadIdx.x;
        __syncthreads();
        const int owner = sm.owner;
        if (owner < 0) break;
        if (owner == (int)threadIdx.x) {
            sm.c_start = start;
            sm.c_len = len;
            sm.c_pred = pred;
            sm.c_out = out;
            len = 0;
        }
        __syncthreads();
        const int s = sm.c_start;
        gather_list<THREADS>(p.col, p.vec_end, s & ~3, s, sm.c_len, sm.c_pred, sm.c_out, threadIdx.x, sink, pol);
    }
    // (2) warp gather of lists >= warp_th
    unsigned wm;
    while ((wm = __ballot_sync(FULL, len >= p.warp_th)) != 0u) {
        const int leader = __ffs(wm) - 1;
        const int s = __shfl_sync(FULL, start, leader);
        const int l = __shfl_sync(FULL, len, leader);
        const int pv = __shfl_sync(FULL, pred, leader);
        const unsigned o = __shfl_sync(FULL, out, leader);
        if ((int)lane_id() == leader) len = 0;
        gather_list<32>(p.col, p.vec_end, s & ~3, s, l, pv, o, lane_id(), sink, pol);
    }
    // (3) scan-based gather of the short lists through shared memory
    constexpr int SCRATCH = Smem<THREADS, MP>::SCRATCH;
    const int my_len = small ? len : 0;
    for (int round = 0; round < small_total; round += SCRATCH) {
        const int lo = max(small_off, round), hi = min(small_off + my_len, round + SCRATCH);
        for (int j = lo; j < hi; j++) {
            sm.gofs[j - round] = start + (j - small_off);
            if (MP) sm.gpred[j - round] = pred;
        }
        __syncthreads();
        const int cnt = min(SCRATCH, small_total - round);
        const int k = threadIdx.x * 4;  // SCRATCH = 4 * THREADS: one pass
        unsigned valid = 0;
        int u[4], pv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            u[j] = -1;
            pv[j] = 0;
            if (k + j < cnt) {
                valid |= 1u << j;
                u[j] = __ldg(p.col + sm.gofs[k + j]);
                if (MP) pv[j] = sm.gpred[k + j];
            }
        }
        sink(valid, u, pv, small_base + unsigned(round + k));
        __syncthreads();
    }
}

// Cuts list [start, start+len) into grid-wide chunks aligned to CHUNK-element
// windows from the 4-aligned start.  Returns false when the chunk table is
// full; the entries it reserved are then written empty and the caller's CTA
// gathers the list itself.
template <int THREADS>
__device__ __forceinline__ bool push_chunks(const BfsParams &p, unsigned *chunk_count, int start, int len, int pred,
                                            unsigned out) {
    constexpr int CH = chunk_edges<THREADS>();
    const int a0 = start & ~3, end = start + len;
    const unsigned nch = unsigned((end - a0 + CH - 1) / CH);
    const unsigned base = atomicAdd(chunk_count, nch);
    const unsigned cap = (unsigned)p.chunk_cap;
    if (base + nch <= cap) {
        for (unsigned c = 0; c < nch; c++) {
            const int ws = a0 + int(c) * CH;
            const int cs = max(ws, start), ce = min(ws + CH, end);
            p.chunks[base + c] = make_int4(cs, ce - cs, pred, int(out + unsigned(cs - start)));
        }
        return true;
    }
    for (unsigned c = base; c < cap && c < base + nch; c++) p.chunks[c] = make_int4(0, 0, 0, 0);
    return false;
}

// Grid-wide phase: CTA b gathers chunks b, b + G, b + 2G, ...
template <int THREADS, class Sink>
__device__ __forceinline__ void gather_chunks(const BfsParams &p, unsigned n, const Sink &sink, uint64_t pol) {
    if (n > (unsigned)p.chunk_cap) n = p.chunk_cap;
    const unsigned G = gridDim.x;
    unsigned k = blockIdx.x;
    int4 cur = k < n ? __ldcg(p.chunks + k) : make_int4(0, 0, 0, 0);
    for (; k < n; k += G) {
        int4 nxt = (k + G < n) ? __ldcg(p.chunks + k + G) : make_int4(0, 0, 0, 0);
        if (cur.y > 0)
            gather_list<THREADS>(p.col, p.vec_end, cur.x & ~3, cur.x, cur.y, cur.z, unsigned(cur.w), threadIdx.x,
                                 sink, pol);
        cur = nxt;
    }
}

// Hands out tiles of the input frontier to CTAs with one atomic each.
template <int THREADS, bool MP>
__device__ __forceinline__ unsigned next_tile(unsigned *steal, Smem<THREADS, MP> &sm) {
    __syncthreads();
    if (threadIdx.x == 0) sm.tile = atomicAdd(steal, 1u);
    __syncthreads();
    return sm.tile;
}

// Tile size for a frontier of L elements: at most `most`, small enough that
// there are about two tiles per CTA when the frontier is short.
__device__ __forceinline__ unsigned tile_size(unsigned L, unsigned most) {
    const unsigned G2 = 2u * gridDim.x;
    unsigned t = (L + G2 - 1) / G2;
    return t < 1u ? 1u : (t > most ? most : t);
}

__device__ __forceinline__ void row_range(const BfsParams &p, int v, int &start, int &len) {
    start = __ldg(p.row_offsets + v);
    len = __ldg(p.row_offsets + v + 1) - start;
}

// ---------------------------------------------------------------------------------------
// Level bodies
// ---------------------------------------------------------------------------------------

// Expand-contract tile phase of level `it`: vertex frontier queue[it&1] ->
// discovered vertices in queue[(it+1)&1]; lists >= big_th become chunks counted
// in big[it&3].
template <int THREADS, bool MP>
__device__ void ec_level(const BfsParams &p, int it, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[it & 1];
    DiscoverSink<THREADS, MP> sink{p, sm, p.queue[(it + 1) & 1], &c->qlen[(it + 1) & 3], it + 1};
    const unsigned tv = tile_size(L, THREADS);
    const unsigned ntiles = (L + tv - 1) / tv;
    for (;;) {
        const unsigned tile = next_tile<THREADS, MP>(&c->steal[it & 3], sm);
        if (tile >= ntiles) break;
        const unsigned idx = tile * tv + threadIdx.x;
        int v = -1, start = 0, len = 0;
        if (threadIdx.x < tv && idx < L) {
            v = ld_cg(q_in + idx);
            row_range(p, v, start, len);
            if (len >= p.big_th && push_chunks<THREADS>(p, &c->big[it & 3], start, len, v, 0u)) len = 0;
        }
        int small_total;
        const int small_off = block_exclusive_scan<THREADS>(len < p.warp_th ? len : 0, small_total, sm.warp_tot);
        expand_lists<THREADS, MP>(p, sm, sink, pol, start, len, v, 0u, small_off, small_total, 0u);
    }
}

template <int THREADS, bool MP>
__device__ void ec_chunks(const BfsParams &p, int it, unsigned n, Smem<THREADS, MP> &sm, uint64_t pol) {
    DiscoverSink<THREADS, MP> sink{p, sm, p.queue[(it + 1) & 1], &p.ctr->qlen[(it + 1) & 3], it + 1};
    gather_chunks<THREADS>(p, n, sink, pol);
}

// Expands one list per thread into the edge-frontier queue q_out: a
// two-component block scan sizes the short and the long lists, thread 0
// reserves the tile's output with one atomicAdd (ScanTileWithEnqueue,
// util/scan/cooperative_scan.cuh:173-195), lists >= big_th become chunks with
// their reserved output positions.
template <int THREADS, bool MP>
__device__ __forceinline__ void expand_tile_to_edges(const BfsParams &p, Smem<THREADS, MP> &sm, uint64_t pol,
                                                     int start, int len, int pred, int *q_out, int *pq_out,
                                                     unsigned *qlen_out, unsigned *chunk_count) {
    const bool small = len < p.warp_th;
    int2 total;
    const int2 off =
        block_exclusive_scan2<THREADS>(make_int2(small ? len : 0, small ? 0 : len), total, sm.warp_tot);
    if (threadIdx.x == 0) {
        const unsigned need = unsigned(total.x + total.y);
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
    if (base == NO_SPACE) return;  // uniform: the tile's output is dropped on overflow
    const unsigned out = small ? base + off.x : base + unsigned(total.x) + off.y;
    if (len >= p.big_th && push_chunks<THREADS>(p, chunk_count, start, len, pred, out)) len = 0;
    PositionSink<MP> sink{q_out, pq_out};
    expand_lists<THREADS, MP>(p, sm, sink, pol, start, len, pred, out, off.x, total.x, base);
}

// Loads up to 4 edge-frontier elements of tile `tile` (tile size te) per
// thread, strided by THREADS, and culls them.  Returns the survivors' bits.
template <int THREADS, bool MP>
__device__ __forceinline__ unsigned contract_tile_load(const BfsParams &p, Smem<THREADS, MP> &sm, const int *q_in,
                                                       const int *pq_in, unsigned L, unsigned tile, unsigned te,
                                                       int (&u)[4], int (&pr)[4]) {
    unsigned valid = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const unsigned r = j * THREADS + threadIdx.x;
        const unsigned idx = tile * te + r;
        u[j] = -1;
        pr[j] = 0;
        if (r < te && idx < L) {
            valid |= 1u << j;
            u[j] = ld_cg(q_in + idx);
            if (MP) pr[j] = ld_cg(pq_in + idx);
        }
    }
    return cull4<THREADS, MP>(p, sm, valid, u);
}

// Contract-expand level `it` (contract_expand_atomic/cta.cuh:573-709): edge
// frontier queue[it&1] -> cull, label it -> survivors compacted in shared
// memory -> expanded into queue[(it+1)&1].
template <int THREADS, bool MP>
__device__ void ce_level(const BfsParams &p, int it, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[it & 1];
    const int *pq_in = p.pred_queue[it & 1];
    const unsigned te = tile_size(L, Smem<THREADS, MP>::CTILE);
    const unsigned ntiles = (L + te - 1) / te;
    for (;;) {
        const unsigned tile = next_tile<THREADS, MP>(&c->steal[it & 3], sm);
        if (tile >= ntiles) break;
        int u[4], pr[4];
        const unsigned surv = contract_tile_load<THREADS, MP>(p, sm, q_in, pq_in, L, tile, te, u, pr);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((surv >> j) & 1u) p.labels[u[j]] = MP ? pr[j] : it;
        int nsurv;
        int off = block_exclusive_scan<THREADS>(__popc(surv), nsurv, sm.warp_tot);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((surv >> j) & 1u) sm.surv[off++] = u[j];
        __syncthreads();
        for (int r0 = 0; r0 < nsurv; r0 += THREADS) {
            int v = -1, start = 0, len = 0;
            if (r0 + (int)threadIdx.x < nsurv) {
                v = sm.surv[r0 + threadIdx.x];
                row_range(p, v, start, len);
            }
            expand_tile_to_edges<THREADS, MP>(p, sm, pol, start, len, v, p.queue[(it + 1) & 1],
                                              p.pred_queue[(it + 1) & 1], &c->qlen[(it + 1) & 3], &c->big[it & 3]);
        }
    }
}

// Chunk phase after a level that wrote an edge frontier to queue[out_sel].
template <int THREADS, bool MP>
__device__ void edge_chunks(const BfsParams &p, int out_sel, unsigned n, uint64_t pol) {
    PositionSink<MP> sink{p.queue[out_sel], p.pred_queue[out_sel]};
    gather_chunks<THREADS>(p, n, sink, pol);
}

// Two-phase contract (two_phase/contract_atomic/cta.cuh:494-572): edge frontier
// queue[qi&1] -> cull, label `it` -> compacted vertex frontier queue[(qi+1)&1],
// allocated by a block scan and one atomicAdd per tile.
template <int THREADS, bool MP>
__device__ void tp_contract(const BfsParams &p, int it, int qi, unsigned L, Smem<THREADS, MP> &sm) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[qi & 1];
    const int *pq_in = p.pred_queue[qi & 1];
    int *q_out = p.queue[(qi + 1) & 1];
    const unsigned te = tile_size(L, Smem<THREADS, MP>::CTILE);
    const unsigned ntiles = (L + te - 1) / te;
    for (;;) {
        const unsigned tile = next_tile<THREADS, MP>(&c->steal[qi & 3], sm);
        if (tile >= ntiles) break;
        int u[4], pr[4];
        const unsigned surv = contract_tile_load<THREADS, MP>(p, sm, q_in, pq_in, L, tile, te, u, pr);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((surv >> j) & 1u) p.labels[u[j]] = MP ? pr[j] : it;
        int total;
        int off = block_exclusive_scan<THREADS>(__popc(surv), total, sm.warp_tot);
        if (threadIdx.x == 0) {
            unsigned base = total ? atomicAdd(&c->qlen[(qi + 1) & 3], (unsigned)total) : 0u;
            if ((unsigned long long)base + total > (unsigned long long)p.qcap) {
                atomicOr(&c->error, ERR_OVERFLOW);
                base = NO_SPACE;
            }
            sm.out_base = base;
        }
        __syncthreads();
        const unsigned base = sm.out_base;
        if (base != NO_SPACE) {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if ((surv >> j) & 1u) q_out[base + off++] = u[j];
        }
    }
}

// Two-phase expand (two_phase/expand_atomic/cta.cuh:606-719): vertex frontier
// queue[qi&1] -> edge frontier queue[(qi+1)&1] with predecessors.
template <int THREADS, bool MP>
__device__ void tp_expand(const BfsParams &p, int qi, unsigned L, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int *q_in = p.queue[qi & 1];
    const unsigned tv = tile_size(L, THREADS);
    const unsigned ntiles = (L + tv - 1) / tv;
    for (;;) {
        const unsigned tile = next_tile<THREADS, MP>(&c->steal[qi & 3], sm);
        if (tile >= ntiles) break;
        const unsigned idx = tile * tv + threadIdx.x;
        int v = -1, start = 0, len = 0;
        if (threadIdx.x < tv && idx < L) {
            v = ld_cg(q_in + idx);
            row_range(p, v, start, len);
        }
        expand_tile_to_edges<THREADS, MP>(p, sm, pol, start, len, v, p.queue[(qi + 1) & 1],
                                          p.pred_queue[(qi + 1) & 1], &c->qlen[(qi + 1) & 3], &c->big[qi & 3]);
    }
}

// Ring housekeeping for phase index q: entries that phase q+1 will use start
// from zero.  Done by one thread while no CTA touches them.
__device__ __forceinline__ void ring_prepare(Counters *c, int q) {
    c->qlen[(q + 2) & 3] = 0u;
    c->steal[(q + 1) & 3] = 0u;
    c->big[(q + 1) & 3] = 0u;
}

__device__ __forceinline__ void log_level_start(const BfsParams &p, int idx, unsigned frontier) {
    if (p.levels && idx < p.level_cap) {
        LevelRecord r;
        r.t_start = globaltimer_ns();
        r.t_tiles = 0;
        r.frontier = frontier;
        r.chunks = 0;
        p.levels[idx] = r;
    }
}
__device__ __forceinline__ void log_level_tiles(const BfsParams &p, int idx, unsigned chunks) {
    if (p.levels && idx < p.level_cap) {
        p.levels[idx].t_tiles = globaltimer_ns();
        p.levels[idx].chunks = chunks;
    }
}

template <int THREADS, bool MP>
__device__ __forceinline__ void init_hist(Smem<THREADS, MP> &sm, unsigned flags) {
    if (flags & CULL_HISTORY)
        for (int i = threadIdx.x; i < HIST_SIZE; i += THREADS) sm.hist[i] = -1;
}

__device__ __forceinline__ bool leader() { return blockIdx.x == 0 && threadIdx.x == 0; }

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

// Leaves the loop of a fused kernel (every CTA decides alike: L and the level
// index are the same everywhere after a barrier).
__device__ __forceinline__ bool stop_level_loop(const BfsParams &p, int level, unsigned L) {
    if (L == 0u) return true;
    if (level_limit_hit(level, p.nodes)) {
        if (leader()) atomicOr(&p.ctr->error, ERR_LEVEL_LIMIT);
        return true;
    }
    return false;
}

__device__ __forceinline__ void finish_search(const BfsParams &p, int iteration, int log_idx) {
    if (leader()) {
        p.ctr->iteration = iteration;
        log_level_start(p, log_idx, 0u);  // end-of-search timestamp
        atomicOr(&p.ctr->sticky, ld_relaxed_gpu(&p.ctr->error));
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
        const unsigned L = ld_cg(&c->qlen[it & 3]);
        if (stop_level_loop(p, it, L)) break;
        if (leader()) {
            ring_prepare(c, it);
            c->total_queued += L;
            log_level_start(p, it, L);
        }
        ec_level<THREADS, MP>(p, it, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        const unsigned nch = ld_cg(&c->big[it & 3]);
        if (leader()) log_level_tiles(p, it, nch);
        if (nch) {
            ec_chunks<THREADS, MP>(p, it, nch, sm, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        it++;
    }
    finish_search(p, it, it);
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ce_fused_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int it = 0;
    for (;;) {
        const unsigned L = ld_cg(&c->qlen[it & 3]);
        if (stop_level_loop(p, it, L)) break;
        if (leader()) {
            ring_prepare(c, it);
            c->total_queued += L;
            log_level_start(p, it, L);
        }
        ce_level<THREADS, MP>(p, it, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        const unsigned nch = ld_cg(&c->big[it & 3]);
        if (leader()) log_level_tiles(p, it, nch);
        if (nch) {
            edge_chunks<THREADS, MP>(p, (it + 1) & 1, nch, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        it++;
    }
    finish_search(p, it, it);
}

// Fused two-phase: contract and expand phases alternate across grid barriers
// (the reference's fused two-phase kernel, two_phase/kernel.cuh:60-313, which
// its enactor cannot instantiate, enactor_two_phase.cuh:302).  The level log is
// indexed by phase (2 * iteration for contract, + 1 for expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_fused_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int it = 0, qi = 0;
    for (;;) {
        unsigned L = ld_cg(&c->qlen[qi & 3]);
        if (stop_level_loop(p, it, L)) break;
        if (leader()) {
            ring_prepare(c, qi);
            c->total_queued += L;
            log_level_start(p, qi, L);
        }
        tp_contract<THREADS, MP>(p, it, qi, L, sm);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        qi++;
        L = ld_cg(&c->qlen[qi & 3]);
        if (L == 0u) break;
        if (leader()) {
            ring_prepare(c, qi);
            log_level_start(p, qi, L);
        }
        tp_expand<THREADS, MP>(p, qi, L, sm, pol);
        if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        const unsigned nch = ld_cg(&c->big[qi & 3]);
        if (leader()) log_level_tiles(p, qi, nch);
        if (nch) {
            edge_chunks<THREADS, MP>(p, (qi + 1) & 1, nch, pol);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        qi++;
        it++;
    }
    finish_search(p, it, qi + 1);
}

// ---- per-level kernels for the graph-driven (iterative) variants ----------------

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ec_level_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3];
    if (L == 0u || p.ctr->error) return;
    if (leader()) log_level_start(p, it, L);
    ec_level<THREADS, MP>(p, it, L, sm, policy_evict_first());
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ec_chunks_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned n = p.ctr->big[it & 3];
    if (leader()) log_level_tiles(p, it, n);
    if (n == 0u || p.ctr->error) return;
    ec_chunks<THREADS, MP>(p, it, n, sm, policy_evict_first());
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) ce_level_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3];
    if (L == 0u || p.ctr->error) return;
    if (leader()) log_level_start(p, it, L);
    ce_level<THREADS, MP>(p, it, L, sm, policy_evict_first());
}

// Chunk pass after a per-level kernel that wrote an edge frontier: ring index
// q = iteration (contract-expand) or 2 * iteration + 1 (two-phase expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) edge_chunks_kernel(BfsParams p, int two_phase) {
    const int q = two_phase ? p.ctr->cur_it * 2 + 1 : p.ctr->cur_it;
    const unsigned n = p.ctr->big[q & 3];
    if (leader()) log_level_tiles(p, q, n);
    if (n == 0u || p.ctr->error) return;
    edge_chunks<THREADS, MP>(p, (q + 1) & 1, n, policy_evict_first());
}

// Two-phase per-level: qi = 2 * it (contract) and 2 * it + 1 (expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_contract_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it;
    const unsigned L = p.ctr->qlen[qi & 3];
    if (L == 0u || p.ctr->error) return;
    if (leader()) log_level_start(p, qi, L);
    tp_contract<THREADS, MP>(p, it, qi, L, sm);
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS) tp_expand_kernel(BfsParams p) {
    __shared__ Smem<THREADS, MP> sm;
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it + 1;
    const unsigned L = p.ctr->qlen[qi & 3];
    if (L == 0u || p.ctr->error) return;
    if (leader()) log_level_start(p, qi, L);
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
            c->iteration = it;  // the reference leaves after contract without ++
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
        if (!more) log_level_start(p, vq == 0u ? qi + 1 : qi + 2, 0u);
    } else {
        const unsigned next = c->qlen[(it + 1) & 3];
        c->total_queued += c->qlen[it & 3];
        c->iteration = it + 1;
        more = next != 0u;
        c->steal[(it + 1) & 3] = 0u;
        c->big[(it + 1) & 3] = 0u;
        c->qlen[(it + 2) & 3] = 0u;
        if (!more) log_level_start(p, it + 1, 0u);
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
    return kc.mark_pred ? fused_fn_t<true>(kc.threads, kc.strategy) : fused_fn_t<false>(kc.threads, kc.strategy);
}

struct LevelFns {
    KernelFn level_a;  // ec_level / ce_level / tp_contract
    KernelFn level_b;  // ec_chunks / (none) / tp_expand
    void (*edge_chunks)(BfsParams, int);
};

template <int THREADS, bool MP>
static LevelFns level_fns(int strategy) {
    LevelFns f{};
    f.edge_chunks = edge_chunks_kernel<THREADS, MP>;
    switch (strategy) {
    case STRATEGY_EXPAND_CONTRACT:
        f.level_a = ec_level_kernel<THREADS, MP>;
        f.level_b = ec_chunks_kernel<THREADS, MP>;
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
    return kc.mark_pred ? level_fns_t<true>(kc.threads, kc.strategy) : level_fns_t<false>(kc.threads, kc.strategy);
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
        if ((e = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)))
            break;
        LevelFns f = pick_level(kc);
        const int T = kc.threads;
        f.level_a<<<grid, T, 0, cap>>>(p);
        if (kc.strategy == STRATEGY_EXPAND_CONTRACT) {
            f.level_b<<<grid, T, 0, cap>>>(p);
        } else if (kc.strategy == STRATEGY_CONTRACT_EXPAND) {
            f.edge_chunks<<<grid, T, 0, cap>>>(p, 0);
        } else {
            f.level_b<<<grid, T, 0, cap>>>(p);
            f.edge_chunks<<<grid, T, 0, cap>>>(p, 1);
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
        if ((e = cudaLaunchCooperativeKernel((const void *)barrier_timeout_probe_kernel, dim3(grid), dim3(32), args, 0,
                                             nullptr)))
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
