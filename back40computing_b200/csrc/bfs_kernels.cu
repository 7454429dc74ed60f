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
// Work is organised by warps; no level body waits on a CTA-wide barrier.
// Neighbour lists are gathered by the reference's strategies chosen by list
// length (two_phase/expand_atomic/cta.cuh:215-423):
//   * lists >= cta_th are cut, when their vertex is discovered, into chunks of
//     16 * THREADS edges for the NEXT level; there every CTA of the grid takes
//     chunks in turn and streams each with all its threads (CTA-based gather,
//     spread over the grid so a hub never serialises a level);
//   * lists >= warp_th are streamed by one warp (warp-based gather);
//   * shorter lists are packed by a warp prefix sum into a per-warp shared
//     memory window of gather offsets that the warp reads together
//     (scan-based gather).
// CTA and warp gathers use 16-byte loads of column indices with an L2
// evict_first policy, issued one pass ahead of use.  Contract-expand and
// two-phase contract the chunks straight from the column array instead of
// copying hub lists through the edge-frontier queue.
//
// Culling: the visited bitmask is the authority and is updated with atomicOr
// (exact), so each vertex is labelled and expanded once.  Each thread tests 4
// elements at a time: 4 mask loads in flight, then at most 4 atomicOr, then one
// warp-aggregated queue reservation (the reference reserves with one atomic
// per CTA tile, util/scan/cooperative_scan.cuh:173-195).  Optional warp-level
// (__match_any_sync) and per-CTA history-hash culls drop repeats first
// (two_phase/contract_atomic/cta.cuh:276-327).

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>

#include "bfs_kernels.cuh"

namespace b40c_b200 {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WINDOW = 128;      // per-warp scan-gather window (4 per lane)

// Resident CTAs per SM requested from ptxas: 40 warps per SM (48 registers
// per thread); the kernels are bound by memory latency, so resident warps
// matter more than registers.
#define MIN_BLOCKS(threads) (1280 / (threads))

constexpr int OBUF = 256;        // per-warp staging of vertex-queue appends
constexpr int TILE_GRAB = 4;     // warp tiles handed out per atomic

template <bool MP>
struct WarpSmem {
    int gofs[WINDOW];
    int gpred[MP ? WINDOW : 1];
    int surv[WINDOW];
    int obuf[OBUF];
    int opred[MP ? OBUF : 1];    // owners staged with obuf (edge-frontier appends with predecessors)
    unsigned nbuf;
    unsigned raw_n;              // edge-frontier entries this warp's expansions produced in the phase
    unsigned zmark_n;            // bottom-up: vertices without edges this warp marked in the level
    unsigned disc_n;             // direction-optimizing counts of this warp's discoveries
    unsigned long long disc_m;   // in the current level, added to the counters at its end
    unsigned bfound[4];          // bottom-up window scans: vertex 32j + lane found a parent
    unsigned segstart[4];        // bottom-up window scans: window positions where a list starts
};

template <int THREADS, bool MP>
struct Smem {
    WarpSmem<MP> w[THREADS / 32];
    unsigned long long vcache[VCACHE];  // (mask word index << 32) | word value
    LevelCounts lc;
    unsigned flag;
};

// L2 policy of the column stream: evict_first when the column array is large
// next to L2 (it then passes through once per search and must not push out
// the mask, labels and row offsets); evict_normal when the whole graph can
// stay in L2 between searches.
__device__ __forceinline__ uint64_t column_policy(const BfsParams &p) {
    return p.stream_col ? policy_evict_first() : policy_evict_normal();
}

// ---------------------------------------------------------------------------------------
// Culling and enqueueing, 4 elements per thread
// ---------------------------------------------------------------------------------------


// Exact test-and-set of the visited bits of up to 4 vertices (bit j of valid
// marks u[j]).  Returns the bits of the vertices this thread claimed first.
//
// The history cull (the reference's per-CTA history hash of recently seen
// ids, two_phase/contract_atomic/cta.cuh:276-297) is kept here as a
// shared-memory cache of visited-mask words.  Bits are only ever set during a
// search, so a cached word is a lower bound of the true one: a bit set there
// culls the vertex with no global access, a clear bit falls through to the L2
// probe, whose result refreshes the entry.  Hub vertices' words stay cached,
// which keeps their mask lines from becoming L2 hot spots.  The optional warp
// cull (__match_any_sync) drops repeats inside a warp first.
//
// probe: test the mask with an L2 load before claiming (large levels, where
// most elements are already visited and the load spares their atomics); on
// small levels every element the cache does not cull goes straight to
// atomicOr, one round trip less.  With ROWS, the row ranges of the elements
// sent to atomicOr are loaded together with the atomics, and st / ln hold
// those of the claimed elements (0 / 0 otherwise).
template <int THREADS, bool MP, bool ROWS = false>
__device__ __forceinline__ unsigned cull4(const BfsParams &p, Smem<THREADS, MP> &sm, unsigned valid,
                                          const int (&u)[4], bool probe, int (&st)[4], int (&ln)[4]) {
    const bool history = p.cull_flags & CULL_HISTORY;
    if (p.cull_flags & CULL_WARP) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            // Lanes without an element get distinct negative keys so they never match.
            const bool ok = (valid >> j) & 1u;
            const int key = ok ? u[j] : int(0x80000000u | lane_id());
            const unsigned peers = __match_any_sync(FULL, key);
            if (ok && (int)lane_id() != __ffs(peers) - 1) valid &= ~(1u << j);
        }
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
        if (ok && history) {
            const unsigned long long e = sm.vcache[vcache_slot(w[j])];
            if (unsigned(e >> 32) == w[j] && (unsigned(e) & bit[j])) valid &= ~(1u << j);
        }
    }
    unsigned need = valid;
    if (probe) {
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = ((valid >> j) & 1u) ? ld_cg(p.mask + w[j]) : 0u;  // probes in flight
        need = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (((valid >> j) & 1u) && !(m[j] & bit[j])) need |= 1u << j;
    } else {
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = 0u;
    }
    unsigned old[4];
#pragma unroll
    for (int j = 0; j < 4; j++) old[j] = ((need >> j) & 1u) ? atomicOr(p.mask + w[j], bit[j]) : m[j];
    int r0[4], r1[4];
    if (ROWS) {  // issued behind the atomics, before their results are used
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int vv = ((need >> j) & 1u) ? u[j] : 0;
            r0[j] = __ldg(p.row_offsets + vv);
            r1[j] = __ldg(p.row_offsets + vv + 1);
        }
    }
    unsigned claimed = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if ((valid >> j) & 1u) {
            if (!(old[j] & bit[j])) claimed |= 1u << j;
            if (history)
                sm.vcache[vcache_slot(w[j])] = ((unsigned long long)w[j] << 32) | (old[j] | bit[j]);
        }
    }
    if (ROWS) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool c = (claimed >> j) & 1u;
            st[j] = c ? r0[j] : 0;
            ln[j] = c ? r1[j] - r0[j] : 0;
        }
    }
    return claimed;
}

// The elements a phase's sinks receive: its queue entries (each list of a
// vertex queue counted as avg_list entries) and its chunk tables' edges.
template <int THREADS>
__device__ __forceinline__ unsigned long long phase_work(unsigned L, unsigned avg_list, unsigned nch, unsigned nw) {
    return (unsigned long long)L * avg_list + (unsigned long long)nch * chunk_edges<THREADS>() +
           (unsigned long long)nw * WARP_CHUNK;
}

// Whether a level whose sinks receive about `work` elements probes the mask
// before claiming (cull4): more than 4 elements per thread of the grid.
__device__ __forceinline__ bool probe_level(unsigned long long work) {
    return work > 4ull * blockDim.x * gridDim.x;
}

// Writes the warp's staged appends to queue q with one atomicAdd (coalesced
// stores).  Called by all lanes together.
template <bool MP>
__device__ __forceinline__ void warp_flush(WarpSmem<MP> &ws, unsigned n, int *q, unsigned *qlen, long long qcap,
                                           unsigned *err) {
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(qlen, n);
    base = __shfl_sync(FULL, base, 0);
    for (unsigned i = lane_id(); i < n; i += 32) {
        const unsigned long long pos = (unsigned long long)base + i;
        if (pos < (unsigned long long)qcap) q[pos] = ws.obuf[i];
        else atomicOr(err, ERR_OVERFLOW);
    }
    __syncwarp();
}

// Stages the flagged elements of every lane (bit j of flags marks u[j]) in the
// warp's buffer; flushes it to queue q when fewer than 128 slots stay free.
// The reference reserves queue space with one atomic per CTA tile
// (util/scan/cooperative_scan.cuh:173-195); here it is one per <= 256
// appends of a warp.  Called by all lanes together.
template <bool MP>
__device__ __forceinline__ void stage4(WarpSmem<MP> &ws, unsigned flags, const int (&u)[4], int *q, unsigned *qlen,
                                       long long qcap, unsigned *err) {
    const unsigned lt = lanemask_lt();
    unsigned total = 0, pre[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        unsigned b = __ballot_sync(FULL, (flags >> j) & 1u);
        pre[j] = total + __popc(b & lt);
        total += __popc(b);
    }
    if (total == 0u) return;  // warp-uniform
    unsigned n = ws.nbuf;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if ((flags >> j) & 1u) ws.obuf[n + pre[j]] = u[j];
    n += total;
    __syncwarp();
    if (n > unsigned(OBUF - WINDOW)) {
        warp_flush(ws, n, q, qlen, qcap, err);
        n = 0;
    }
    if (lane_id() == 0) ws.nbuf = n;
    __syncwarp();
}

// Flushes what the warp still holds; every warp calls it at the end of a phase.
template <bool MP>
__device__ __forceinline__ void stage_drain(WarpSmem<MP> &ws, int *q, unsigned *qlen, long long qcap, unsigned *err) {
    const unsigned n = ws.nbuf;
    if (n) warp_flush(ws, n, q, qlen, qcap, err);
    if (lane_id() == 0) ws.nbuf = 0;
    __syncwarp();
}

__device__ __forceinline__ void row_range(const BfsParams &p, int v, int &start, int &len) {
    start = __ldg(p.row_offsets + v);
    len = __ldg(p.row_offsets + v + 1) - start;
}

// Reserves, with one atomicAdd for the whole warp, chunk-table entries for the
// lists flagged in sel (nc[j] chunks of CH edges for list j of this lane, n in
// all) and writes their descriptors: windows of CH elements from the list's
// 4-aligned start, clipped to the list.  Returns sel, or 0 when the table
// would overflow (the reserved entries are then written empty and the lists
// stay with their lanes).  Called by all lanes together.
template <int CH>
__device__ __forceinline__ unsigned place_tier(int4 *table, unsigned *count, int cap, unsigned sel, int n,
                                               const int (&nc)[4], const int (&st)[4], const int (&ln)[4],
                                               const int (&pr)[4]) {
    const int incl = warp_inclusive_scan(n);
    const unsigned total = (unsigned)__shfl_sync(FULL, incl, 31);
    if (total == 0u) return 0u;  // warp-uniform
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(count, total);
    base = __shfl_sync(FULL, base, 0);
    unsigned my = base + unsigned(incl - n);
    if ((unsigned long long)base + total <= (unsigned long long)cap) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((sel >> j) & 1u) {
                const int a0 = st[j] & ~3, end = st[j] + ln[j];
                for (int c = 0; c < nc[j]; c++) {
                    const int ws = a0 + c * CH;
                    const int cs = max(ws, st[j]), ce = min(ws + CH, end);
                    table[my++] = make_int4(cs, ce - cs, pr[j], 0);
                }
            }
        }
        return sel;
    }
    for (unsigned c = my; c < (unsigned)cap && c < my + unsigned(n); c++) table[c] = make_int4(0, 0, 0, 0);
    return 0u;
}

// Places up to 4 lists per lane (bit j of has marks list j: start st[j],
// length ln[j], owner pr[j]) for phase q_next by length: lists >= cta_th are
// cut into CTA chunks, lists >= warp_th into warp chunks; shorter lists stay
// with their lanes.  Returns the bits of the lists placed in a chunk table.
// Called by all lanes together.
// c: the counters the chunk counts go to (p.ctr, or a narrow launch's copy).
template <int THREADS>
__device__ __forceinline__ unsigned place4(const BfsParams &p, int q_next, unsigned has, const int (&st)[4],
                                           const int (&ln)[4], const int (&pr)[4], Counters *c) {
    constexpr int CH = chunk_edges<THREADS>();
    unsigned cta = 0, wrp = 0;
    int ncta = 0, nw = 0, nc[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        nc[j] = 0;
        if ((has >> j) & 1u) {
            const int span = st[j] + ln[j] - (st[j] & ~3);
            if (ln[j] >= p.cta_th) {
                cta |= 1u << j;
                nc[j] = (span + CH - 1) / CH;
                ncta += nc[j];
            } else if (ln[j] >= p.warp_th) {
                wrp |= 1u << j;
                nc[j] = (span + WARP_CHUNK - 1) / WARP_CHUNK;
                nw += nc[j];
            }
        }
    }
    if (!__any_sync(FULL, (cta | wrp) != 0u)) return 0u;
    const int nq = q_next & 1;
    unsigned placed = place_tier<CH>(p.chunks[nq], &c->big[q_next & 3], p.chunk_cap, cta, ncta, nc, st, ln, pr);
    placed |= place_tier<WARP_CHUNK>(p.wchunks[nq], &c->wch[q_next & 3], p.wchunk_cap, wrp, nw, nc, st, ln, pr);
    return placed;
}
template <int THREADS>
__device__ __forceinline__ unsigned place4(const BfsParams &p, int q_next, unsigned has, const int (&st)[4],
                                           const int (&ln)[4], const int (&pr)[4]) {
    return place4<THREADS>(p, q_next, has, st, ln, pr, p.ctr);
}

// ---------------------------------------------------------------------------------------
// Gather strategies
// ---------------------------------------------------------------------------------------

// Grid-wide chunk phase: CTA b streams chunks b, b + G, b + 2G, ... of table.
template <int THREADS, class Sink>
__device__ __forceinline__ void gather_chunks(const BfsParams &p, const int4 *table, unsigned n, const Sink &sink,
                                              uint64_t pol) {
    if (n > (unsigned)p.chunk_cap) n = p.chunk_cap;
    const unsigned G = gridDim.x;
    unsigned k = blockIdx.x;
    int4 cur = k < n ? __ldcg(table + k) : make_int4(0, 0, 0, 0);
    for (; k < n; k += G) {
        int4 nxt = (k + G < n) ? __ldcg(table + k + G) : make_int4(0, 0, 0, 0);
        if (cur.y > 0) gather_list<THREADS>(p.col, p.vec_end, cur.x, cur.y, cur.z, 0u, threadIdx.x, sink, pol);
        cur = nxt;
    }
}

// Warp w of the grid is warp w / gridDim.x of CTA w % gridDim.x: consecutive
// work items (tiles, steps, runs) go to different CTAs, and so to different
// SMs, so a level with few items still spreads over the whole GPU instead of
// crowding the issue slots and memory pipes of the first few SMs.
__device__ __forceinline__ int global_warp() { return int((threadIdx.x >> 5) * gridDim.x + blockIdx.x); }
__device__ __forceinline__ int grid_warps() { return int(gridDim.x * (blockDim.x >> 5)); }

// Warp chunk phase: warp w of the grid streams warp chunks w, w + W, ...
template <class Sink>
__device__ __forceinline__ void gather_wchunks(const BfsParams &p, const int4 *table, unsigned n, const Sink &sink,
                                               uint64_t pol) {
    if (n > (unsigned)p.wchunk_cap) n = p.wchunk_cap;
    const unsigned W = grid_warps();
    unsigned k = global_warp();
    int4 cur = k < n ? __ldcg(table + k) : make_int4(0, 0, 0, 0);
    for (; k < n; k += W) {
        int4 nxt = (k + W < n) ? __ldcg(table + k + W) : make_int4(0, 0, 0, 0);
        if (cur.y > 0) gather_list<32>(p.col, p.vec_end, cur.x, cur.y, cur.z, 0u, lane_id(), sink, pol);
        cur = nxt;
    }
}

// Both chunk tables of a phase.  When their slices of 128 edges (one 16-byte
// load per lane) number no more than the grid's warps, every warp takes one
// slice: a small level then finishes in one pass instead of the 4 passes a
// CTA or warp needs for a whole chunk.  Otherwise CTAs stream CTA chunks and
// warps stream warp chunks.
template <int THREADS, class Sink>
__device__ __forceinline__ void gather_chunk_tables(const BfsParams &p, const int4 *ctable, unsigned nch,
                                                    const int4 *wtable, unsigned nw, const Sink &sink,
                                                    uint64_t pol) {
    constexpr unsigned SLICE = 128;
    constexpr unsigned CS = chunk_edges<THREADS>() / SLICE, WS = WARP_CHUNK / SLICE;
    if (nch > (unsigned)p.chunk_cap) nch = p.chunk_cap;
    if (nw > (unsigned)p.wchunk_cap) nw = p.wchunk_cap;
    const unsigned long long slices = (unsigned long long)nch * CS + (unsigned long long)nw * WS;
    if (slices > (unsigned long long)grid_warps()) {
        gather_chunks<THREADS>(p, ctable, nch, sink, pol);
        gather_wchunks(p, wtable, nw, sink, pol);
        return;
    }
    const unsigned w = global_warp();
    if (w >= slices) return;
    const int4 ch = w < nch * CS ? __ldcg(ctable + w / CS) : __ldcg(wtable + (w - nch * CS) / WS);
    const unsigned k = w < nch * CS ? w % CS : (w - nch * CS) % WS;
    const int a0 = (ch.x & ~3) + int(k * SLICE);
    const int s0 = max(a0, ch.x), e0 = min(a0 + int(SLICE), ch.x + ch.y);
    if (e0 > s0) gather_list<32>(p.col, p.vec_end, s0, e0 - s0, ch.z, 0u, lane_id(), sink, pol);
}

// ---- window gathers of up to 4 lists per lane ------------------------------------------
// The lists a warp holds (bit j of has marks list j of a lane: column entries
// [st[j], st[j] + ln[j]), owner pr[j]) are laid out one after the other, list
// 0 of every lane, then list 1, and so on (list_layout gives each list's first
// position o[j] and returns the warp's total).  The warp streams that layout in
// windows of WINDOW positions, 4 per lane (position 32m + lane of the window).
// Each list that reaches into a window writes one segment record (its column
// base relative to the window) and marks the position where it starts in a
// bitmap; a position finds its list by counting the starts up to it.  Lists
// of any length take the same path, consecutive lanes read consecutive column
// entries, and a window costs one column load per lane and element whatever
// the mix of lengths.

__device__ __forceinline__ unsigned list_layout(unsigned has, const int (&ln)[4], int (&o)[4]) {
    unsigned total = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int l = ((has >> j) & 1u) ? ln[j] : 0;
        const int incl = warp_inclusive_scan(l);
        o[j] = int(total) + incl - l;
        total += unsigned(__shfl_sync(FULL, incl, 31));
    }
    return total;
}

// Window [w0, w0 + WINDOW) of the layout: e[m] = the column index at window
// position 32m + lane (own[m] its list's owner), for positions below cw =
// min(WINDOW, total - w0); returns cw.  Ends with the warp's shared records
// read, so the next window may rewrite them after a __syncwarp.
template <bool MP>
__device__ __forceinline__ int window_entries(WarpSmem<MP> &ws, unsigned has, const int (&st)[4],
                                              const int (&ln)[4], const int (&pr)[4], const int (&o)[4],
                                              unsigned w0, unsigned total, int (&e)[4], int (&own)[4]) {
    const int lane = lane_id();
    if (lane < 4) ws.segstart[lane] = 0u;
    __syncwarp();
    int nseg = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int l = ((has >> j) & 1u) ? ln[j] : 0;
        const bool seg = l > 0 && o[j] < int(w0) + WINDOW && o[j] + l > int(w0);
        const unsigned b = __ballot_sync(FULL, seg);
        if (seg) {
            const int k = nseg + __popc(b & lanemask_lt());
            const int s0 = max(o[j], int(w0)) - int(w0);
            ws.gofs[k] = st[j] - o[j] + int(w0);
            if (MP) ws.gpred[k] = pr[j];
            atomicOr(&ws.segstart[s0 >> 5], 1u << (s0 & 31));
        }
        nseg += __popc(b);
    }
    __syncwarp();
    const int cw = min(WINDOW, int(total - w0));
    unsigned sw[4];
    int before[4];  // segment starts in the words before word m
#pragma unroll
    for (int m = 0; m < 4; m++) {
        sw[m] = ws.segstart[m];
        before[m] = m ? before[m - 1] + __popc(sw[m - 1]) : 0;
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int idx = m * 32 + lane;
        const int k = before[m] + __popc(sw[m] & ((2u << lane) - 1u)) - 1;
        e[m] = idx < cw ? ws.gofs[k] + idx : -1;
        own[m] = (MP && idx < cw) ? ws.gpred[k] : 0;
    }
    return cw;
}

// Positional gather: one atomicAdd on qlen_out reserves room in q_out for every
// entry of the warp's lists, which are then written at their layout positions
// (the owners into pq_out when MP).  Called by all lanes together.
template <bool MP>
__device__ __forceinline__ void gather_positional4(const BfsParams &p, WarpSmem<MP> &ws, unsigned has,
                                                   const int (&st)[4], const int (&ln)[4], const int (&pr)[4],
                                                   int *q_out, int *pq_out, unsigned *qlen_out, uint64_t pol) {
    int o[4];
    const unsigned total = list_layout(has, ln, o);
    if (total == 0u) return;  // warp-uniform
    unsigned base = 0;
    for (unsigned w0 = 0; w0 < total; w0 += WINDOW) {
        int e[4], own[4], x[4];
        window_entries<MP>(ws, has, st, ln, pr, o, w0, total, e, own);
#pragma unroll
        for (int m = 0; m < 4; m++) x[m] = e[m] >= 0 ? ldg_stream(p.col + e[m], pol) : 0;
        if (w0 == 0) {  // the reservation's round trip overlaps the first window's loads
            if (lane_id() == 0) {
                base = atomicAdd(qlen_out, total);
                if ((unsigned long long)base + total > (unsigned long long)p.qcap) {
                    atomicOr(&p.ctr->error, ERR_OVERFLOW);
                    base = 0xffffffffu;
                }
            }
            base = __shfl_sync(FULL, base, 0);
            if (base == 0xffffffffu) return;  // warp-uniform: output dropped on overflow
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            if (e[m] >= 0) {
                const unsigned pos = base + w0 + unsigned(m * 32) + lane_id();
                q_out[pos] = x[m];
                if (MP) pq_out[pos] = own[m];
            }
        }
        __syncwarp();
    }
}

// Sink-based gather: every window's elements go to sink (valid bits, 4
// elements and their owners per lane).  Called by all lanes together.
template <bool MP, class Sink>
__device__ __forceinline__ void gather_windows4(const BfsParams &p, WarpSmem<MP> &ws, unsigned has,
                                                const int (&st)[4], const int (&ln)[4], const int (&pr)[4],
                                                const Sink &sink, uint64_t pol) {
    int o[4];
    const unsigned total = list_layout(has, ln, o);
    for (unsigned w0 = 0; w0 < total; w0 += WINDOW) {
        int e[4], own[4], x[4];
        window_entries<MP>(ws, has, st, ln, pr, o, w0, total, e, own);
        unsigned valid = 0;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            x[m] = e[m] >= 0 ? ldg_stream(p.col + e[m], pol) : -1;
            if (e[m] >= 0) valid |= 1u << m;
        }
        __syncwarp();
        sink(valid, x, own, 0u);
    }
}

// Frontier vertices per lane of a warp tile: 4 (tiles of WINDOW vertices, row
// ranges and lists of four vertices per lane in flight together) once a level
// has at least two such tiles per warp of the grid, else 1 (tiles of 32), so
// that a small level still gives every warp of the grid a tile.
__device__ __forceinline__ unsigned vertices_per_lane(unsigned L) {
    return (unsigned long long)L >= 2ull * WINDOW * unsigned(grid_warps()) ? 4u : 1u;
}

// Loads the frontier vertices of warp tile t (per vertices per lane, tile
// size 32 * per) from q_in; bit j of the result marks v[j].
__device__ __forceinline__ unsigned load_tile(const int *q_in, unsigned L, unsigned t, unsigned per, int (&v)[4]) {
    unsigned sel = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const unsigned idx = t * 32u * per + unsigned(j) * 32u + lane_id();
        v[j] = -1;
        if (unsigned(j) < per && idx < L) {
            v[j] = ld_cg(q_in + idx);
            sel |= 1u << j;
        }
    }
    return sel;
}

// Row ranges of up to 4 vertices per lane (bit j of sel marks v[j]): every
// load is issued before any is used (an unselected slot reads row 0, a line
// the warp shares).  Sets has to the selected vertices with edges.
__device__ __forceinline__ unsigned row_ranges4(const BfsParams &p, unsigned sel, const int (&v)[4], int (&st)[4],
                                                int (&ln)[4]) {
    int r0[4], r1[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int vv = ((sel >> j) & 1u) ? v[j] : 0;
        r0[j] = __ldg(p.row_offsets + vv);
        r1[j] = __ldg(p.row_offsets + vv + 1);
    }
    unsigned has = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        st[j] = r0[j];
        ln[j] = ((sel >> j) & 1u) ? r1[j] - r0[j] : 0;
        if (ln[j] > 0) has |= 1u << j;
    }
    return has;
}

// Warp tiles handed out per atomic: several when there are many per warp.
__device__ __forceinline__ unsigned tile_grab(unsigned ntiles) {
    return ntiles >= unsigned(grid_warps()) * 16u ? TILE_GRAB : 1u;
}

__device__ __forceinline__ unsigned warp_next_tile(unsigned *steal) {
    unsigned t = 0;
    if (lane_id() == 0) t = atomicAdd(steal, 1u);
    return __shfl_sync(FULL, t, 0);
}

// Next run of tiles for a warp that finished run r: the first W runs go one
// per warp without atomics (a small phase then costs no counter traffic);
// runs beyond them are handed out by the steal counter.
__device__ __forceinline__ unsigned next_run(unsigned nruns, unsigned *steal) {
    const unsigned W = grid_warps();
    return nruns > W ? W + warp_next_tile(steal) : nruns;
}

// ---------------------------------------------------------------------------------------
// Sinks: what happens to each gathered element.  Called by every lane of a
// warp together with up to 4 elements per lane; bit j of valid marks u[j];
// output positions (edge-frontier queues) are out0 + j.
// ---------------------------------------------------------------------------------------

// Edge-frontier appends with their owners (predecessor labels): as stage4,
// with the owners staged beside the ids and written to pq at the same
// positions.  Called by all lanes together.
template <bool MP>
__device__ __forceinline__ void pair_flush(WarpSmem<MP> &ws, unsigned n, int *q, int *pq, unsigned *qlen,
                                           long long qcap, unsigned *err) {
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(qlen, n);
    base = __shfl_sync(FULL, base, 0);
    for (unsigned i = lane_id(); i < n; i += 32) {
        const unsigned long long pos = (unsigned long long)base + i;
        if (pos < (unsigned long long)qcap) {
            q[pos] = ws.obuf[i];
            if (MP) pq[pos] = ws.opred[i];
        } else {
            atomicOr(err, ERR_OVERFLOW);
        }
    }
    __syncwarp();
}

template <bool MP>
__device__ __forceinline__ void stage_pairs4(WarpSmem<MP> &ws, unsigned flags, const int (&u)[4], const int (&pr)[4],
                                             int *q, int *pq, unsigned *qlen, long long qcap, unsigned *err) {
    const unsigned lt = lanemask_lt();
    unsigned total = 0, pre[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        unsigned b = __ballot_sync(FULL, (flags >> j) & 1u);
        pre[j] = total + __popc(b & lt);
        total += __popc(b);
    }
    if (total == 0u) return;  // warp-uniform
    unsigned n = ws.nbuf;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if ((flags >> j) & 1u) {
            ws.obuf[n + pre[j]] = u[j];
            if (MP) ws.opred[n + pre[j]] = pr[j];
        }
    }
    n += total;
    __syncwarp();
    if (n > unsigned(OBUF - WINDOW)) {
        pair_flush(ws, n, q, pq, qlen, qcap, err);
        n = 0;
    }
    if (lane_id() == 0) ws.nbuf = n;
    __syncwarp();
}

// Adds the lengths of a lane's lists (bit j of has marks ln[j]) to the warp's
// raw edge-frontier count of the phase; flush_raw adds the warp's count to
// the counters once, at the phase's end.
__device__ __forceinline__ void count_raw(unsigned *raw_n, unsigned has, const int (&ln)[4]) {
    unsigned l = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) l += ((has >> j) & 1u) ? unsigned(ln[j]) : 0u;
    l = __reduce_add_sync(FULL, l);
    if (lane_id() == 0) *raw_n += l;
}
template <bool MP>
__device__ __forceinline__ void flush_raw(const BfsParams &p, WarpSmem<MP> &ws, int q) {
    if (lane_id() == 0) {
        if (ws.raw_n) atomicAdd(&p.ctr->raw[q & 3], ws.raw_n);
        ws.raw_n = 0u;
    }
    __syncwarp();
}

// The edge frontier a phase starts from: its raw count when the phase before
// counted it (INSTRUMENT, or a culling expand), else its queue entries plus
// the edges of its chunk tables.
template <int THREADS>
__device__ __forceinline__ unsigned long long level_edges(const LevelCounts &lc) {
    const unsigned long long est = (unsigned long long)lc.L + (unsigned long long)lc.nch * chunk_edges<THREADS>() +
                                   (unsigned long long)lc.nw * WARP_CHUNK;
    return est > lc.raw ? est : (unsigned long long)lc.raw;
}

// Whether a two-phase expand culls while it gathers, by the edge frontier raw
// its level started from: on large levels (more than 4 entries per thread of
// the grid, the hybrid's saturation point) most gathered neighbours are
// already visited -- the contract phase before the barrier has set every bit
// of the level -- and dropping them early saves their queue traffic and
// contraction; on small levels the extra probe only lengthens the level's
// dependent chain.
__device__ __forceinline__ bool gather_cull(unsigned long long raw) {
    return raw > 4ull * blockDim.x * gridDim.x;
}

// The gather-time cull of the edge-frontier strategies: a gathered neighbour
// whose visited bit is already set (seen in the CTA's history cache of mask
// words, else by one L2 probe of the mask) can never be contracted, so it is
// dropped instead of being written to the next edge frontier, read back and
// culled there.  The bit is only read here; the next phase's contraction
// still claims every remaining vertex with atomicOr.  Entries outside [0,
// nodes) raise ERR_BAD_VERTEX here, as contraction would.
template <int THREADS, bool MP>
struct FilterSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int *q_out;
    int *pq_out;
    unsigned *qlen_out;

    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&own)[4],
                                               unsigned) const {
        const bool history = p.cull_flags & CULL_HISTORY;
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
            if (ok && history) {
                const unsigned long long e = sm.vcache[vcache_slot(w[j])];
                if (unsigned(e >> 32) == w[j] && (unsigned(e) & bit[j])) valid &= ~(1u << j);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = ((valid >> j) & 1u) ? ld_cg(p.mask + w[j]) : 0u;
        unsigned keep = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((valid >> j) & 1u) {
                if (!(m[j] & bit[j])) keep |= 1u << j;
                if (history) sm.vcache[vcache_slot(w[j])] = ((unsigned long long)w[j] << 32) | m[j];
            }
        }
        stage_pairs4(sm.w[threadIdx.x >> 5], keep, u, own, q_out, pq_out, qlen_out, p.qcap, &p.ctr->error);
    }
    __device__ __forceinline__ void drain() const {
        WarpSmem<MP> &ws = sm.w[threadIdx.x >> 5];
        const unsigned n = ws.nbuf;
        if (n) pair_flush(ws, n, q_out, pq_out, qlen_out, p.qcap, &p.ctr->error);
        if (lane_id() == 0) ws.nbuf = 0;
        __syncwarp();
    }
};

// Direction-optimizing counts: a warp sums its discoveries (n vertices with
// deg edges per lane) in shared memory during a level and adds them to the
// counters of phase q once, at the level's end (one atomic pair per warp;
// an atomic per discovery group would make the counters a hot spot).
template <bool MP>
__device__ __forceinline__ void count_discovered(WarpSmem<MP> &ws, int n, long long deg) {
    // Degrees of distinct vertices of one graph sum to less than its int32
    // edge count, so 32-bit warp reductions (one instruction each) suffice.
    const unsigned nt = __reduce_add_sync(0xffffffffu, unsigned(n));
    const unsigned dt = __reduce_add_sync(0xffffffffu, unsigned(deg));
    if (lane_id() == 0 && nt) {
        ws.disc_n += nt;
        ws.disc_m += (unsigned long long)dt;
    }
}
template <bool MP>
__device__ __forceinline__ void flush_discovered(const BfsParams &p, WarpSmem<MP> &ws, int q) {
    if (lane_id() == 0) {
        if (ws.disc_n) {
            atomicAdd(&p.ctr->nf[q & 3], ws.disc_n);
            atomicAdd(&p.ctr->mf[q & 3], ws.disc_m);
        }
        // Bottom-up levels count the vertices without edges they mark per warp
        // (one atomic per step on one address made that address a hot spot).
        if (ws.zmark_n) atomicAdd(&p.ctr->zmarked, ws.zmark_n);
        ws.disc_n = 0u;
        ws.disc_m = 0ull;
        ws.zmark_n = 0u;
    }
    __syncwarp();
}

// Expand-contract: mark and label each neighbour at discovery (label it+1,
// expand_contract_atomic/cta.cuh:181-218).  A discovered vertex's list becomes
// CTA or warp chunks of the next level when it is long enough; the other
// vertices go to the next vertex frontier.
template <int THREADS, bool MP>
struct DiscoverSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int *q_out;
    unsigned *qlen_out;
    int label;  // it + 1; also the phase whose inputs the discovered lists become
    bool probe;  // cull4's mask probe before claiming (probe_level)

    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pred)[4],
                                               unsigned) const {
        int st[4], ln[4];
        const unsigned disc = cull4<THREADS, MP, true>(p, sm, valid, u, probe, st, ln);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((disc >> j) & 1u) p.labels[u[j]] = MP ? pred[j] : label;
        if (p.do_alpha)
            count_discovered(sm.w[threadIdx.x >> 5], __popc(disc), (long long)ln[0] + ln[1] + ln[2] + ln[3]);
        const unsigned enq = disc & ~place4<THREADS>(p, label, disc, st, ln, u);
        stage4(sm.w[threadIdx.x >> 5], enq, u, q_out, qlen_out, p.qcap, &p.ctr->error);
    }
    __device__ __forceinline__ void drain() const {
        stage_drain(sm.w[threadIdx.x >> 5], q_out, qlen_out, p.qcap, &p.ctr->error);
        if (p.do_alpha) flush_discovered(p, sm.w[threadIdx.x >> 5], label);
    }
};

// Contract-expand survivors' short lists staged per warp before their gather:
// the warp's append buffer obuf (idle in contract-expand) holds up to LSTAGE
// lists as three arrays (starts, lengths, owners), and one positional gather
// -- one queue reservation -- serves them all.  A reservation per contracted
// tile (most tiles of a large level contract one or two vertices) made the
// queue's length counter the level's hot spot.
constexpr int LSTAGE = 64;
static_assert(3 * LSTAGE <= OBUF, "the list stage lives in obuf");

// Gathers the staged lists (two per lane) into queue q_out and empties the
// stage.  Called by all lanes together.
template <bool MP>
__device__ __forceinline__ void flush_lists(const BfsParams &p, WarpSmem<MP> &ws, int *q_out, int *pq_out,
                                         unsigned *qlen_out, uint64_t pol) {
    const unsigned n = ws.nbuf;
    if (n == 0u) return;  // warp-uniform
    int st[4] = {0, 0, 0, 0}, ln[4] = {0, 0, 0, 0}, pr[4] = {0, 0, 0, 0};
    unsigned has = 0;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const unsigned k = unsigned(j) * 32u + lane_id();
        if (k < n) {
            st[j] = ws.obuf[k];
            ln[j] = ws.obuf[LSTAGE + k];
            pr[j] = ws.obuf[2 * LSTAGE + k];
            has |= 1u << j;
        }
    }
    __syncwarp();
    if (lane_id() == 0) ws.nbuf = 0u;
    __syncwarp();
    gather_positional4<MP>(p, ws, has, st, ln, pr, q_out, pq_out, qlen_out, pol);
}

// Contract-expand: cull and label the edge-frontier elements (label it,
// contract_expand_atomic/cta.cuh:264-304), then expand the survivors at once:
// long lists become CTA or warp chunks of the next level (contracted from the
// column array there), the others are copied into the next edge frontier by
// one window gather of all the warp's survivors.  (No gather-time cull here:
// the neighbours gathered in a level are mostly vertices that other warps
// contract in the same level, whose bits are not set yet.)
template <int THREADS, bool MP>
struct ContractExpandSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int it;  // depth label of the contracted vertices
    int q;   // ring phase: reads queue[q&1], writes queue[(q+1)&1] and ring slot q+1
    uint64_t pol;
    bool probe;  // cull4's mask probe before claiming (probe_level)

    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pred)[4],
                                               unsigned) const {
        // The survivors' row ranges come with the claims (loaded together with
        // the atomics), then their lists: long ones to the next phase's chunk
        // tables, the rest gathered by the warp into the next edge frontier.
        int st[4], ln[4];
        const unsigned surv = cull4<THREADS, MP, true>(p, sm, valid, u, probe, st, ln);
        if (!__any_sync(FULL, surv != 0u)) return;
        unsigned has = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (ln[j] > 0) has |= 1u << j;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((surv >> j) & 1u) p.labels[u[j]] = MP ? pred[j] : it;
        WarpSmem<MP> &ws = sm.w[threadIdx.x >> 5];
        if (p.count_raw) count_raw(&ws.raw_n, has, ln);
        const unsigned placed = place4<THREADS>(p, q + 1, has, st, ln, u);
        const unsigned rest = has & ~placed;
        const int nq = (q + 1) & 1;
        // Stage the short lists; gather when the stage would overflow.
        const unsigned lt = lanemask_lt();
        unsigned total = 0, pre[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const unsigned b = __ballot_sync(FULL, (rest >> j) & 1u);
            pre[j] = total + __popc(b & lt);
            total += __popc(b);
        }
        if (total == 0u) return;  // warp-uniform
        unsigned n = ws.nbuf;
        if (n + total > unsigned(LSTAGE)) {
            flush_lists(p, ws, p.queue[nq], p.pred_queue[nq], &p.ctr->qlen[(q + 1) & 3], pol);
            n = 0u;
        }
        if (total > unsigned(LSTAGE)) {  // more than a stage's worth in one tile: gather them now
            gather_positional4<MP>(p, ws, rest, st, ln, u, p.queue[nq], p.pred_queue[nq], &p.ctr->qlen[(q + 1) & 3],
                                   pol);
            return;
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if ((rest >> j) & 1u) {
                const unsigned k = n + pre[j];
                ws.obuf[k] = st[j];
                ws.obuf[LSTAGE + k] = ln[j];
                ws.obuf[2 * LSTAGE + k] = u[j];
            }
        }
        __syncwarp();
        if (lane_id() == 0) ws.nbuf = n + total;
        __syncwarp();
    }
    // Gathers the warp's staged lists and adds its raw count to the counters;
    // every warp calls it at the phase's end.
    __device__ __forceinline__ void drain() const {
        const int nq = (q + 1) & 1;
        flush_lists(p, sm.w[threadIdx.x >> 5], p.queue[nq], p.pred_queue[nq], &p.ctr->qlen[(q + 1) & 3], pol);
        flush_raw(p, sm.w[threadIdx.x >> 5], q + 1);
    }
};

// Two-phase contract: cull and label (iteration it), then append the survivors
// to the vertex frontier (two_phase/contract_atomic/cta.cuh:494-572).
template <int THREADS, bool MP>
struct ContractSink {
    const BfsParams &p;
    Smem<THREADS, MP> &sm;
    int *q_out;
    unsigned *qlen_out;
    int it;
    bool probe;  // cull4's mask probe before claiming (probe_level)

    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pred)[4],
                                               unsigned) const {
        int st[4], ln[4];
        const unsigned surv = cull4<THREADS, MP>(p, sm, valid, u, probe, st, ln);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if ((surv >> j) & 1u) p.labels[u[j]] = MP ? pred[j] : it;
        stage4(sm.w[threadIdx.x >> 5], surv, u, q_out, qlen_out, p.qcap, &p.ctr->error);
    }
    __device__ __forceinline__ void drain() const {
        stage_drain(sm.w[threadIdx.x >> 5], q_out, qlen_out, p.qcap, &p.ctr->error);
    }
};

// ---------------------------------------------------------------------------------------
// Phase bodies.  Phase q reads queue[q&1] (qlen[q&3] entries) and chunks[q&1]
// (big[q&3] entries) and writes queue[(q+1)&1] / chunks[(q+1)&1].
// ---------------------------------------------------------------------------------------

// Expand-contract level it: vertex frontier -> discovered vertices labelled it+1.
// Warp tiles of frontier vertices (vertices_per_lane): their row ranges are
// loaded together and their lists streamed by one window gather into the
// discovery sink.
template <int THREADS, bool MP>
__device__ void ec_level(const BfsParams &p, int it, unsigned L, unsigned nch, unsigned nwch, Smem<THREADS, MP> &sm,
                         uint64_t pol) {
    Counters *c = p.ctr;
    const int nq = (it + 1) & 1;
    // a vertex queue's lists are shorter than warp_th; count 16 entries each
    DiscoverSink<THREADS, MP> sink{p, sm, p.queue[nq], &c->qlen[(it + 1) & 3], it + 1,
                                   probe_level(phase_work<THREADS>(L, 16u, nch, nwch))};
    gather_chunk_tables<THREADS>(p, p.chunks[it & 1], nch, p.wchunks[it & 1], nwch, sink, pol);
    WarpSmem<MP> &ws = sm.w[threadIdx.x >> 5];
    const int *q_in = p.queue[it & 1];
    const unsigned per = vertices_per_lane(L);
    const unsigned ntiles = (L + 32u * per - 1) / (32u * per);
    const unsigned grab = tile_grab(ntiles);
    const unsigned nruns = (ntiles + grab - 1) / grab;
    for (unsigned r = global_warp(); r < nruns; r = next_run(nruns, &c->steal[it & 3])) {
        const unsigned t0 = r * grab;
        for (unsigned t = t0; t < t0 + grab && t < ntiles; t++) {
            int v[4], st[4], ln[4];
            const unsigned sel = load_tile(q_in, L, t, per, v);
            const unsigned has = row_ranges4(p, sel, v, st, ln);
            gather_windows4<MP>(p, ws, has, st, ln, v, sink, pol);
        }
    }
    sink.drain();
}

// Bottom-up level it of direction-optimizing BFS (Beamer, Asanovic and
// Patterson, "Direction-Optimizing Breadth-First Search", SC 2012): every
// unvisited vertex looks for a neighbour at depth it, and the first one found
// makes it a depth-(it+1) vertex.
//
// A warp takes BU_WORDS consecutive mask words per step; lane j owns vertex
// 32w + j of each word w and probes its heaviest neighbour first (from a
// dense per-vertex array); the lists of the vertices that probe does not
// settle are then scanned by the whole warp, a window of entries at a time,
// until each finds a parent or ends.  A word has one writer in the level, so
// its new bits are a plain store.  Vertices without edges are
// marked visited but never labelled: on a symmetric graph no list leads to
// them, and later bottom-up levels skip them.  The discovered vertices are
// counted and placed for level it+1 exactly as top-down discovery places
// them, so either direction can run next.  With predecessor labels the
// probe tests a snapshot of the visited mask instead (see bu_step).
constexpr int BU_WORDS = 4;  // = the 4 lists per lane that place4 and stage4 take
static_assert(BU_WORDS == 4, "bottom-up steps hand 4 vertices per lane to place4 / stage4");

// A bottom-up step's inputs staged in shared memory: the row offsets of its
// 128 vertices (129 used, whole 16-byte units copied), their heaviest-neighbour
// keys and the step's 4 visited-mask words.  Each warp keeps two, so that the
// bulk copies of its next step run while it works on the current one.
struct alignas(16) BuStage {
    int off[32 * BU_WORDS + 4];
    unsigned long long key[32 * BU_WORDS];
    unsigned mask[BU_WORDS];
};
struct alignas(16) WarpStage {
    BuStage buf[2];
    unsigned long long bar[2];  // mbarriers: bar[b] completes when buf[b] has landed
};

// One bottom-up step: visited-mask words w0 .. w0 + BU_WORDS - 1.
template <int THREADS, bool MP>
__device__ __forceinline__ void bu_step(const BfsParams &p, int it, unsigned w0, unsigned nwords, WarpSmem<MP> &ws,
                                        int *q_out, unsigned *qlen_out, const BuStage *sg) {
    Counters *c = p.ctr;
    const int lane = lane_id();
    unsigned mw[BU_WORDS];
#pragma unroll
    for (int j = 0; j < BU_WORDS; j++) mw[j] = w0 + j < nwords ? (sg ? sg->mask[j] : ld_cg(p.mask + w0 + j)) : FULL;
    bool any_open = false;
#pragma unroll
    for (int j = 0; j < BU_WORDS; j++) any_open |= mw[j] != FULL;
    if (!any_open) return;  // warp-uniform
    int v[BU_WORDS], st[BU_WORDS], ln[BU_WORDS];
    int par[MP ? BU_WORDS : 1];  // predecessor labels: the parent found
    unsigned open = 0, scan = 0, found = 0;
    // Every load of a phase is issued before any result is tested, and a lane
    // without work reads entry 0 (a line the whole warp shares) instead of
    // branching around its load: a load behind a branch, or behind a possible
    // atomic, would wait for the one before it, and the rounds are bound by
    // memory latency.
    int r0[BU_WORDS], r1[BU_WORDS];
    unsigned long long hk[BU_WORDS];  // heaviest neighbour: (degree << 32) | id, 0 = none
#pragma unroll
    for (int j = 0; j < BU_WORDS; j++) {
        v[j] = int((w0 + j) * 32u) + lane;
        if (v[j] < p.nodes && !((mw[j] >> lane) & 1u)) open |= 1u << j;
        if (sg) {  // staged: the step's slice, read from shared memory
            r0[j] = sg->off[j * 32 + lane];
            r1[j] = sg->off[j * 32 + lane + 1];
            hk[j] = p.heavy ? sg->key[j * 32 + lane] : 0ull;
        } else {
            const int vv = ((open >> j) & 1u) ? v[j] : 0;
            r0[j] = __ldg(p.row_offsets + vv);
            r1[j] = __ldg(p.row_offsets + vv + 1);
            hk[j] = p.heavy ? __ldg(p.heavy + vv) : 0ull;
        }
    }
#pragma unroll
    for (int j = 0; j < BU_WORDS; j++) {
        st[j] = r0[j];
        ln[j] = ((open >> j) & 1u) ? r1[j] - r0[j] : 0;
    }
    // Probes are ordinary (L1-cached) label loads: the depth-it labels they
    // look for were written before the level's grid barrier, whose
    // release/acquire orders them before these loads; labels written during
    // this level are it+1 and never match.  With predecessor labels the probe
    // reads the snapshot of the visited mask taken at the level's start: a
    // visited neighbour of an unvisited vertex has depth exactly it
    // (symmetric graph).
    //
    // First each vertex probes its heaviest neighbour, read from a dense
    // per-vertex array (coalesced); only the vertices it does not settle read
    // their list, whose first entry is a scattered DRAM access.
    {
        unsigned hact = 0;
        int hp[BU_WORDS];
#pragma unroll
        for (int j = 0; j < BU_WORDS; j++) {
            const unsigned x = unsigned(hk[j]);
            const bool a = ((open >> j) & 1u) && ln[j] > 0 && hk[j] != 0ull && x < (unsigned)p.nodes;
            if (a) hact |= 1u << j;
            const unsigned xs = a ? x : 0u;
            if constexpr (MP) hp[j] = int(__ldca(p.mask_snap + (xs >> 5)));
            else hp[j] = __ldca(p.labels + xs);
        }
#pragma unroll
        for (int j = 0; j < BU_WORDS; j++) {
            if ((hact >> j) & 1u) {
                const unsigned x = unsigned(hk[j]);
                if constexpr (MP) {
                    if (((unsigned)hp[j] >> (x & 31u)) & 1u) {
                        found |= 1u << j;
                        par[j] = int(x);
                    }
                } else {
                    if (hp[j] == it) found |= 1u << j;
                }
            }
            // a list of one entry was settled by the probe of that entry
            if (((open >> j) & 1u) && !((found >> j) & 1u) && ln[j] > int((hact >> j) & 1u)) scan |= 1u << j;
        }
    }
    // The lists the heaviest neighbour did not settle are scanned by the whole
    // warp in windows of WINDOW entries (4 per lane): every unsettled vertex
    // lays its next entries, in vertex order, into the warp's window, so
    // consecutive lanes read consecutive column entries (coalesced loads) and
    // a window's probes all go out at once.  A vertex whose parent turns up
    // takes no further entries.  A step then costs about one window (one
    // column load and one probe in sequence) instead of a round per pair of
    // entries of its longest list.  Entry 0 of the column array exists
    // whenever some lane has a list to scan.
    if (__any_sync(FULL, scan != 0u)) {
        int done[BU_WORDS] = {0, 0, 0, 0};
        unsigned bad = 0;
        if (lane < BU_WORDS) ws.bfound[lane] = 0u;
        __syncwarp();
        for (;;) {
            int excl[BU_WORDS], rem[BU_WORDS], total = 0;
#pragma unroll
            for (int j = 0; j < BU_WORDS; j++) {
                // at most a window's worth per vertex counts, so sums stay small
                rem[j] = ((scan >> j) & 1u) ? min(ln[j] - done[j], WINDOW) : 0;
                const int incl = warp_inclusive_scan(rem[j]);
                excl[j] = total + incl - rem[j];
                total += __shfl_sync(FULL, incl, 31);
            }
            if (total == 0) break;  // warp-uniform
            // Each vertex with entries in the window starts a segment there:
            // segment k (in vertex order) records its column base and owner,
            // and a bitmap marks the window position where it starts, so a
            // position finds its segment by counting the starts up to it.
            if (lane < BU_WORDS) ws.segstart[lane] = 0u;
            __syncwarp();
            int nseg = 0;
#pragma unroll
            for (int j = 0; j < BU_WORDS; j++) {
                const bool seg = rem[j] > 0 && excl[j] < WINDOW;
                const unsigned b = __ballot_sync(FULL, seg);
                if (seg) {
                    const int k = nseg + __popc(b & lanemask_lt());
                    ws.gofs[k] = st[j] + done[j] - excl[j];
                    ws.surv[k] = j * 32 + lane;
                    atomicOr(&ws.segstart[excl[j] >> 5], 1u << (excl[j] & 31));
                    done[j] += min(rem[j], WINDOW - excl[j]);
                }
                nseg += __popc(b);
            }
            __syncwarp();
            const int cw = min(WINDOW, total);
            unsigned sw[BU_WORDS];
            int before[BU_WORDS];  // segment starts in the words before word w
#pragma unroll
            for (int w = 0; w < BU_WORDS; w++) {
                sw[w] = ws.segstart[w];
                before[w] = w ? before[w - 1] + __popc(sw[w - 1]) : 0;
            }
            int x[4], own[4], pb[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int idx = m * 32 + lane;  // word m of the bitmap, bit lane
                const int k = before[m] + __popc(sw[m] & ((2u << lane) - 1u)) - 1;
                const bool in = idx < cw;
                x[m] = __ldg(p.col + (in ? ws.gofs[k] + idx : 0));
                own[m] = in ? ws.surv[k] : -1;
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const bool a = own[m] >= 0 && (unsigned)x[m] < (unsigned)p.nodes;
                if (own[m] >= 0 && !a) bad = 1u;
                const unsigned xs = a ? (unsigned)x[m] : 0u;
                if constexpr (MP) pb[m] = int(__ldca(p.mask_snap + (xs >> 5)));
                else pb[m] = __ldca(p.labels + xs);
                if (!a) own[m] = -1;
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                if (own[m] < 0) continue;
                const unsigned xu = (unsigned)x[m];
                bool hit;
                if constexpr (MP) hit = ((unsigned)pb[m] >> (xu & 31u)) & 1u;
                else hit = pb[m] == it;
                if (hit) {
                    atomicOr(&ws.bfound[own[m] >> 5], 1u << (own[m] & 31));
                    if constexpr (MP) ws.gpred[own[m]] = int(xu);  // any parent found will do
                }
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < BU_WORDS; j++) {
                if (((scan >> j) & 1u) && ((ws.bfound[j] >> lane) & 1u)) {
                    found |= 1u << j;
                    if constexpr (MP) par[j] = ws.gpred[j * 32 + lane];
                }
                if (((found >> j) & 1u) || done[j] >= ln[j]) scan &= ~(1u << j);
            }
            __syncwarp();
        }
        if (bad) atomicOr(&c->error, ERR_BAD_VERTEX);
    }
    int nfound = 0;
    long long dfound = 0;
#pragma unroll
    for (int j = 0; j < BU_WORDS; j++) {
        const bool f = (found >> j) & 1u;
        const unsigned fb = __ballot_sync(FULL, f);
        const unsigned zb = __ballot_sync(FULL, ((open >> j) & 1u) && ln[j] == 0);
        if (lane == 0 && (fb | zb)) __stcg(p.mask + w0 + j, mw[j] | fb | zb);
        if (lane == 0 && zb) ws.zmark_n += unsigned(__popc(zb));  // added to the counters once, at the level's end
        if (f) {
            p.labels[v[j]] = MP ? par[j] : it + 1;
            nfound++;
            dfound += ln[j];
        }
    }
    count_discovered(ws, nfound, dfound);
    const unsigned placed = place4<THREADS>(p, it + 1, found, st, ln, v);
    stage4(ws, found & ~placed, v, q_out, qlen_out, p.qcap, &c->error);
}

// Copies the visited mask into mask_snap (predecessor-label bottom-up
// levels probe the copy); a grid barrier must follow before it is read.
__device__ __forceinline__ void snapshot_mask(const BfsParams &p) {
    const unsigned nwords = (unsigned(p.nodes) + 31u) >> 5;
    for (unsigned w = blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += gridDim.x * blockDim.x)
        p.mask_snap[w] = ld_cg(p.mask + w);
}

// Issues the bulk copies of bottom-up step `step` into stage buffer b (lane 0
// of the warp).  Copy sizes are whole 16-byte units, clamped to the padded
// ends of the arrays (ROW_PAD, HEAVY_PAD, MASK_PAD_BYTES).  The mask words
// were written by generic stores in earlier levels; the proxy fence orders
// those writes, which the level's grid barrier made visible to this thread,
// before the bulk reads.  Within a bottom-up level no other step writes the
// step's words.
__device__ __forceinline__ void bu_prefetch(const BfsParams &p, unsigned step, WarpStage *stg, int b) {
    if (lane_id() == 0) {
        const long long v0 = (long long)step * (32 * BU_WORDS);
        const long long n = p.nodes;
        const unsigned offs = unsigned(min((long long)(32 * BU_WORDS + 4), n + 1 + ROW_PAD - v0)) & ~3u;
        const unsigned keys = p.heavy ? unsigned(min((long long)(32 * BU_WORDS), n + HEAVY_PAD - v0)) & ~1u : 0u;
        fence_proxy_async_global();
        mbar_arrive_expect_tx(&stg->bar[b], offs * 4u + keys * 8u + 16u);
        bulk_copy_g2s(stg->buf[b].off, p.row_offsets + v0, offs * 4u, &stg->bar[b]);
        if (keys) bulk_copy_g2s(stg->buf[b].key, p.heavy + v0, keys * 8u, &stg->bar[b]);
        bulk_copy_g2s(stg->buf[b].mask, p.mask + step * BU_WORDS, 16u, &stg->bar[b]);
    }
}

// Waits, with the grid barrier's time limit, for stage buffer b's copies;
// phase holds the parity each buffer completes next.  Returns false, with
// ERR_BARRIER_TIMEOUT raised, when the limit passed (warp-uniform).
__device__ __forceinline__ bool bu_stage_wait(const BfsParams &p, WarpStage *stg, int b, unsigned &phase) {
    const unsigned parity = (phase >> b) & 1u;
    bool ok = mbar_try_wait(&stg->bar[b], parity);
    if (!ok) {
        const unsigned long long t0 = globaltimer_ns();
        while (!(ok = mbar_try_wait(&stg->bar[b], parity)))
            if (globaltimer_ns() - t0 > p.wait_ns) break;
    }
    ok = __all_sync(FULL, ok);
    if (ok) phase ^= 1u << b;
    else if (lane_id() == 0) atomicOr(&p.ctr->error, ERR_BARRIER_TIMEOUT);
    return ok;
}

// open: an estimate of the vertices still unvisited.  stg (a warp's stage
// buffers, or NULL) stages each step's row offsets, keys and mask words one
// step ahead with bulk copies; phase is their mbarriers' parity state.
template <int THREADS, bool MP>
__device__ void bu_level(const BfsParams &p, int it, Smem<THREADS, MP> &sm, unsigned open, WarpStage *stg,
                         unsigned &phase) {
    Counters *c = p.ctr;
    int *q_out = p.queue[(it + 1) & 1];
    unsigned *qlen_out = &c->qlen[(it + 1) & 3];
    WarpSmem<MP> &ws = sm.w[threadIdx.x >> 5];
    const unsigned nwords = (unsigned(p.nodes) + 31u) >> 5;
    const unsigned nsteps = (nwords + BU_WORDS - 1) / BU_WORDS;
    const unsigned W = grid_warps();
    // While many vertices are open, steps go one per warp, then to whichever
    // warp is free (a step's cost depends on how long its lists scan, so a
    // static split leaves most warps waiting at the level's barrier for a few
    // slow ones); a warp asks for its next step when it starts one, hiding the
    // atomic's latency.  Once fewer than a quarter are open, most steps are
    // cheap and alike, and a static interleave spares the counter its atomics.
    const bool dynamic = nsteps > W && (unsigned long long)open * 4ull > (unsigned long long)p.nodes;
    if (!stg) {
        for (unsigned step = global_warp(); step < nsteps;) {
            unsigned nxt = 0;
            if (dynamic && lane_id() == 0) nxt = atomicAdd(&c->steal[it & 3], 1u);
            bu_step<THREADS, MP>(p, it, step * BU_WORDS, nwords, ws, q_out, qlen_out, nullptr);
            step = dynamic ? W + __shfl_sync(FULL, nxt, 0) : step + W;
        }
    } else {
        // Two steps in hand: cur (being worked on, in buf b) and nxt (its
        // copies in flight into buf b ^ 1).  The step after nxt is asked for
        // while cur runs and staged into buf b once cur is done.
        unsigned cur = global_warp(), nxt = nsteps;
        int b = 0;
        if (cur < nsteps) {
            bu_prefetch(p, cur, stg, 0);
            unsigned t = 0;
            if (dynamic && lane_id() == 0) t = atomicAdd(&c->steal[it & 3], 1u);
            nxt = dynamic ? W + __shfl_sync(FULL, t, 0) : cur + W;
            if (nxt < nsteps) bu_prefetch(p, nxt, stg, 1);
        }
        while (cur < nsteps) {
            unsigned t = 0;
            const bool more = nxt < nsteps;
            if (more && dynamic && lane_id() == 0) t = atomicAdd(&c->steal[it & 3], 1u);
            if (!bu_stage_wait(p, stg, b, phase)) {
                // Abandon the level: wait (bounded again) for the copies still
                // in flight into the other buffer, then leave.
                if (more) bu_stage_wait(p, stg, b ^ 1, phase);
                break;
            }
            bu_step<THREADS, MP>(p, it, cur * BU_WORDS, nwords, ws, q_out, qlen_out, &stg->buf[b]);
            unsigned nxt2 = nsteps;
            if (more) nxt2 = dynamic ? W + __shfl_sync(FULL, t, 0) : nxt + W;
            if (nxt2 < nsteps) bu_prefetch(p, nxt2, stg, b);
            cur = nxt;
            nxt = nxt2;
            b ^= 1;
        }
    }
    stage_drain(ws, q_out, qlen_out, p.qcap, &c->error);
    flush_discovered(p, ws, it + 1);
}

// Edge-frontier phase input: warp tiles of 128 elements (4 per lane,
// coalesced), statically interleaved over the grid's warps.
template <bool MP, class Sink>
__device__ __forceinline__ void edge_tiles(const int *q_in, const int *pq_in, unsigned L, const Sink &sink) {
    const unsigned ntiles = (L + WINDOW - 1) / WINDOW;
    const unsigned W = grid_warps();
    for (unsigned t = global_warp(); t < ntiles; t += W) {
        unsigned valid = 0;
        int u[4], pr[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const unsigned idx = t * WINDOW + j * 32 + lane_id();
            u[j] = -1;
            pr[j] = 0;
            if (idx < L) {
                valid |= 1u << j;
                u[j] = ld_cg(q_in + idx);
                if (MP) pr[j] = ld_cg(pq_in + idx);
            }
        }
        sink(valid, u, pr, 0u);
    }
}

// Contract-expand level it in ring phase q (contract_expand_atomic/cta.cuh:573-709);
// q == it except in the hybrid kernel, whose two-phase levels take two phases.
template <int THREADS, bool MP>
__device__ void ce_level(const BfsParams &p, int it, int q, unsigned L, unsigned nch, unsigned nwch,
                         Smem<THREADS, MP> &sm, uint64_t pol) {
    ContractExpandSink<THREADS, MP> sink{p, sm, it, q, pol, probe_level(phase_work<THREADS>(L, 1u, nch, nwch))};
    gather_chunk_tables<THREADS>(p, p.chunks[q & 1], nch, p.wchunks[q & 1], nwch, sink, pol);
    edge_tiles<MP>(p.queue[q & 1], p.pred_queue[q & 1], L, sink);
    sink.drain();
}

// Two-phase contract, phase qi = 2 * it.
template <int THREADS, bool MP>
__device__ void tp_contract(const BfsParams &p, int it, int qi, unsigned L, unsigned nch, unsigned nwch,
                            Smem<THREADS, MP> &sm, uint64_t pol) {
    ContractSink<THREADS, MP> sink{p, sm, p.queue[(qi + 1) & 1], &p.ctr->qlen[(qi + 1) & 3], it,
                                   probe_level(phase_work<THREADS>(L, 1u, nch, nwch))};
    gather_chunk_tables<THREADS>(p, p.chunks[qi & 1], nch, p.wchunks[qi & 1], nwch, sink, pol);
    edge_tiles<MP>(p.queue[qi & 1], p.pred_queue[qi & 1], L, sink);
    sink.drain();
}

// Two-phase expand, phase qi = 2 * it + 1 (two_phase/expand_atomic/cta.cuh:606-719):
// warp tiles of frontier vertices (vertices_per_lane); long lists become
// chunks of the next phase, the others are streamed by one window gather per
// tile through the gather-time cull into the next edge frontier.
template <int THREADS, bool MP>
__device__ void tp_expand(const BfsParams &p, int qi, unsigned L, bool cull, Smem<THREADS, MP> &sm, uint64_t pol) {
    Counters *c = p.ctr;
    const int nq = (qi + 1) & 1;
    WarpSmem<MP> &ws = sm.w[threadIdx.x >> 5];
    const FilterSink<THREADS, MP> out{p, sm, p.queue[nq], p.pred_queue[nq], &c->qlen[(qi + 1) & 3]};
    const int *q_in = p.queue[qi & 1];
    const unsigned per = vertices_per_lane(L);
    const unsigned ntiles = (L + 32u * per - 1) / (32u * per);
    const unsigned grab = tile_grab(ntiles);
    const unsigned nruns = (ntiles + grab - 1) / grab;
    for (unsigned r = global_warp(); r < nruns; r = next_run(nruns, &c->steal[qi & 3])) {
        const unsigned t0 = r * grab;
        for (unsigned t = t0; t < t0 + grab && t < ntiles; t++) {
            int v[4], st[4], ln[4];
            const unsigned sel = load_tile(q_in, L, t, per, v);
            const unsigned has = row_ranges4(p, sel, v, st, ln);
            if (cull || p.count_raw) count_raw(&ws.raw_n, has, ln);
            const unsigned placed = place4<THREADS>(p, qi + 1, has, st, ln, v);
            if (cull)
                gather_windows4<MP>(p, ws, has & ~placed, st, ln, v, out, pol);
            else
                gather_positional4<MP>(p, ws, has & ~placed, st, ln, v, p.queue[nq], p.pred_queue[nq],
                                       &c->qlen[(qi + 1) & 3], pol);
        }
    }
    out.drain();
    flush_raw(p, ws, qi + 1);
}

// Ring housekeeping for phase q: the entries phase q+1 writes start at zero.
// Done by one thread while no CTA touches them.
__device__ __forceinline__ void ring_prepare(Counters *c, int q) {
    c->qlen[(q + 2) & 3] = 0u;
    c->big[(q + 2) & 3] = 0u;
    c->wch[(q + 2) & 3] = 0u;
    c->raw[(q + 2) & 3] = 0u;
    c->nf[(q + 2) & 3] = 0u;
    c->mf[(q + 2) & 3] = 0ull;
    c->steal[(q + 1) & 3] = 0u;
}

__device__ __forceinline__ void log_phase(const BfsParams &p, int idx, unsigned frontier, unsigned chunks,
                                          unsigned wchunks, unsigned bottom_up = 0u) {
    if (p.levels && idx < p.level_cap) {
        LevelRecord r;
        r.t_start = globaltimer_ns();
        r.frontier = frontier;
        r.chunks = chunks;
        r.wchunks = wchunks;
        r.bottom_up = bottom_up;
        p.levels[idx] = r;
    }
}

// Level log: the time the last CTA finished phase idx's work, taken when every
// warp of the CTA is done (before the phase's grid barrier).
__device__ __forceinline__ void log_work_end(const BfsParams &p, int idx) {
    if (p.levels && idx < p.level_cap) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(&p.levels[idx].t_work_end, globaltimer_ns());
    }
}

template <int THREADS, bool MP>
__device__ __forceinline__ void init_hist(Smem<THREADS, MP> &sm, unsigned flags) {
    if (lane_id() == 0) {
        sm.w[threadIdx.x >> 5].nbuf = 0;
        sm.w[threadIdx.x >> 5].raw_n = 0;
        sm.w[threadIdx.x >> 5].zmark_n = 0;
        sm.w[threadIdx.x >> 5].disc_n = 0;
        sm.w[threadIdx.x >> 5].disc_m = 0;
    }
    __syncwarp();
    if (flags & CULL_HISTORY) {
        // Tag 0xffffffff matches no mask word (word indices stay below 2^27).
        for (int i = threadIdx.x; i < VCACHE; i += THREADS) sm.vcache[i] = ~0ull << 32;
        __syncthreads();
    }
}

// The thread that does a fused kernel's per-level bookkeeping (ring entries,
// statistics, level log): lane 0 of CTA 0's last warp, which takes tiles only
// when a level has more than (warps per CTA - 1) * grid of them, so that the
// bookkeeping's round trips stay off the warp that takes a small level's
// first tile.
__device__ __forceinline__ bool leader() { return blockIdx.x == 0 && threadIdx.x == blockDim.x - 32; }

// INSTRUMENT duty (the reference's KernelRuntimeStats MarkStart / MarkStop,
// b40c/util/kernel_runtime_stats.cuh): thread 0 of each CTA sums the time from
// a level's start to the moment all its warps finished the level's work.
struct BusyClock {
    unsigned long long busy = 0, t0 = 0;
    __device__ __forceinline__ void start(const BfsParams &p) {
        if (p.cta_busy && threadIdx.x == 0) t0 = globaltimer_ns();
    }
    __device__ __forceinline__ void stop(const BfsParams &p) {
        if (!p.cta_busy) return;
        __syncthreads();
        if (threadIdx.x == 0) busy += globaltimer_ns() - t0;
    }
    __device__ __forceinline__ void flush(const BfsParams &p) const {
        if (p.cta_busy && threadIdx.x == 0) p.cta_busy[blockIdx.x] = busy;
    }
};

// The kernels keep Smem in dynamic shared memory (it can exceed the 48 KB
// static limit at 512 threads); launches pass sizeof(Smem<THREADS, MP>).
template <int THREADS, bool MP>
__device__ __forceinline__ Smem<THREADS, MP> &kernel_smem() {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    return *reinterpret_cast<Smem<THREADS, MP> *>(dyn_smem);
}

// ---------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------

// Per-search initialisation: counters and barrier to zero, the source in the
// first frontier.  Expand-contract labels and marks the source here (as
// expand_contract_atomic/kernel.cuh:291-326); the edge-frontier strategies
// label it when they contract it at iteration 0, with predecessor -2.
__global__ void search_init_kernel(BfsParams p, int strategy, int mark_pred, int cta_chunk) {
    Counters *c = p.ctr;
    unsigned *w = reinterpret_cast<unsigned *>(c);
    constexpr int WORDS = int(offsetof(Counters, sticky) / 4);  // everything but the sticky error
    for (int i = threadIdx.x; i < WORDS; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x != 0) return;
    c->raw[0] = 1u;  // the first edge frontier is the source
    if (strategy == STRATEGY_EXPAND_CONTRACT) {
        p.labels[p.src] = mark_pred ? -2 : 0;
        p.mask[unsigned(p.src) >> 5] |= 1u << (unsigned(p.src) & 31u);
        // The source's list is level 0's input, placed by length like any
        // discovered vertex's list.
        int start, len;
        row_range(p, p.src, start, len);
        c->nf[0] = 1u;
        c->mf[0] = (unsigned long long)len;
        const int a0 = start & ~3, span = start + len - a0;
        const bool cta = len >= p.cta_th, wrp = !cta && len >= p.warp_th;
        const int CH = cta ? cta_chunk : WARP_CHUNK;
        const int nch = (span + CH - 1) / CH;
        if ((cta || wrp) && nch <= (cta ? p.chunk_cap : p.wchunk_cap)) {
            int4 *table = cta ? p.chunks[0] : p.wchunks[0];
            for (int k = 0; k < nch; k++) {
                const int ws = a0 + k * CH;
                const int cs = max(ws, start), ce = min(ws + CH, start + len);
                table[k] = make_int4(cs, ce - cs, p.src, 0);
            }
            if (cta) c->big[0] = unsigned(nch);
            else c->wch[0] = unsigned(nch);
            return;
        }
    } else if (mark_pred) {
        p.pred_queue[0][0] = -2;
    }
    c->qlen[0] = 1u;
    p.queue[0][0] = p.src;
}

// Whether a fused kernel's level loop ends (every CTA decides alike: the
// counters and the level index are the same everywhere after a barrier).
__device__ __forceinline__ bool stop_level_loop(const BfsParams &p, int level, unsigned work) {
    if (work == 0u) return true;
    if (level_limit_hit(level, p.nodes)) {
        if (leader()) atomicOr(&p.ctr->error, ERR_LEVEL_LIMIT);
        return true;
    }
    return false;
}

__device__ __forceinline__ void finish_search(const BfsParams &p, int iteration, int log_idx) {
    if (leader()) {
        p.ctr->iteration = iteration;
        log_phase(p, log_idx, 0u, 0u, 0u);  // end-of-search marker
        atomicOr(&p.ctr->sticky, ld_relaxed_gpu(&p.ctr->error));
    }
}

// Direction of the next level (Beamer et al., SC 2012): top-down turns
// bottom-up once the frontier's edges mf exceed the unvisited vertices' edges
// / alpha, and bottom-up turns back once the frontier holds fewer than
// nodes / beta vertices and is shrinking.  Every CTA keeps the same state and
// reads the same counters after a barrier, so all take the same direction.
struct DirectionChoice {
    unsigned long long explored = 0;  // degrees summed over the vertices visited so far
    unsigned visited = 0;             // vertices visited so far
    unsigned prev_nf = 0;
    bool bottom_up = false;

    __device__ __forceinline__ bool next(const BfsParams &p, unsigned nf, unsigned long long mf) {
        explored += mf;
        visited += nf;
        const unsigned long long total = (unsigned long long)p.edges;
        const unsigned long long unexplored = total > explored ? total - explored : 0ull;
        if (!bottom_up) bottom_up = mf * p.do_alpha > unexplored;
        else bottom_up = !((unsigned long long)nf * p.do_beta < (unsigned long long)p.nodes && nf < prev_nf);
        prev_nf = nf;
        return bottom_up;
    }
    // The state handed from a narrow launch to the full-grid one.
    __device__ __forceinline__ void store(Counters *c) const {
        c->dir_explored = explored;
        c->dir_visited = visited;
        c->dir_prev_nf = prev_nf;
        c->dir_bottom_up = bottom_up ? 1u : 0u;
    }
    __device__ __forceinline__ void load(const Counters *c) {
        explored = __ldcg(&c->dir_explored);
        visited = __ldcg(&c->dir_visited);
        prev_nf = __ldcg(&c->dir_prev_nf);
        bottom_up = __ldcg(&c->dir_bottom_up) != 0u;
    }
};

// The counts a fused kernel's first phase starts from, read once per CTA and
// shared through shared memory (a load per thread would send every warp of
// the grid to the same few L2 lines).  Later phases get theirs from the grid
// barrier before them (next_counts), in the waiting thread's last round trip.
template <int THREADS, bool MP>
__device__ __forceinline__ LevelCounts read_counts(Counters *c, int q, bool dir, Smem<THREADS, MP> &sm) {
    if (threadIdx.x == 0) sm.lc = load_counts(c, q, dir);
    __syncthreads();
    return sm.lc;
}

// Dynamic shared memory of the expand-contract kernel: Smem, then one
// WarpStage per warp when they fit without lowering the kernel's occupancy
// (MIN_BLOCKS CTAs per SM in the SM's 228 KB, 1 KB reserved per CTA).
template <int THREADS, bool MP>
__host__ __device__ constexpr size_t ec_stage_offset() { return (sizeof(Smem<THREADS, MP>) + 15) & ~size_t(15); }
template <int THREADS, bool MP>
__host__ __device__ constexpr bool stage_fits() {
    return (ec_stage_offset<THREADS, MP>() + sizeof(WarpStage) * (THREADS / 32) + 1024) * MIN_BLOCKS(THREADS) <=
           228u * 1024u;
}
template <int THREADS, bool MP>
__host__ __device__ constexpr size_t ec_smem_bytes() {
    return stage_fits<THREADS, MP>() ? ec_stage_offset<THREADS, MP>() + sizeof(WarpStage) * (THREADS / 32)
                                     : sizeof(Smem<THREADS, MP>);
}

// Adds a warp's discovered-vertex degree sum to mf[q] of counters in shared
// memory (a narrow launch's copy) as a 32-bit add on the low word: degrees
// of distinct vertices of one graph sum to less than its int32 edge count, so
// no carry reaches the high word.
__device__ __forceinline__ void add_mf_low(Counters *c, int q, unsigned m) {
    atomicAdd(reinterpret_cast<unsigned *>(&c->mf[q & 3]), m);  // little-endian: the low word
}

// Expand-contract top-down level of a narrow launch, written for latency (as
// ce_narrow_level): frontier vertex i goes to lane i % 32 of warp i / 32
// (warps numbered across the cluster's CTAs).  The lane reads its vertex's
// row range and takes its list (shorter than warp_th: longer ones are in the
// chunk tables, which hand the level to the full grid) 4 entries at a time:
// the 4 claims go out together, each claimed neighbour's row range loaded
// behind its atomic; a discovered vertex is labelled it + 1, its list placed
// by length (place4: a long one makes the next level the full grid's), and
// the warp reserves queue room for the rest with one atomicAdd.  c: the
// level counters (the narrow launch's copy in shared memory).  Labels, queue
// contents (in another order) and counts are ec_level's.
template <int THREADS, bool MP>
__device__ void ec_narrow_level(const BfsParams &p, Counters *c, int it, unsigned L) {
    const int *q_in = p.queue[it & 1];
    int *q_out = p.queue[(it + 1) & 1];
    unsigned *qlen_out = &c->qlen[(it + 1) & 3];
    const int label = it + 1;
    const unsigned W = unsigned(grid_warps());
    const unsigned lane = lane_id(), lt = lanemask_lt();
    unsigned dn = 0, dm = 0;  // this lane's discovered vertices and their degree sum
    for (unsigned w = unsigned(global_warp()); w * 32u < L; w += W) {
        const unsigned i = w * 32u + lane;
        const bool ok = i < L;
        const int u = ok ? ld_cg(q_in + i) : 0;
        const int r0 = ok ? __ldg(p.row_offsets + u) : 0;
        const int len = ok ? __ldg(p.row_offsets + u + 1) - r0 : 0;
        for (int k0 = 0; __any_sync(FULL, k0 < len); k0 += 4) {
            int v[4];
            unsigned valid = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                v[j] = k0 + j < len ? __ldg(p.col + r0 + k0 + j) : 0;
                if (k0 + j < len) {
                    if ((unsigned)v[j] < (unsigned)p.nodes) valid |= 1u << j;
                    else atomicOr(&c->error, ERR_BAD_VERTEX);
                }
            }
            unsigned old[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const unsigned bit = 1u << ((unsigned)v[j] & 31u);
                old[j] = ((valid >> j) & 1u) ? atomicOr(p.mask + ((unsigned)v[j] >> 5), bit) : bit;
            }
            int st[4], ln[4];
            unsigned disc = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {  // row ranges issued behind the atomics
                const bool vj = (valid >> j) & 1u;
                st[j] = vj ? __ldg(p.row_offsets + v[j]) : 0;
                const int r1 = vj ? __ldg(p.row_offsets + v[j] + 1) : 0;
                const bool claimed = vj && !(old[j] & (1u << ((unsigned)v[j] & 31u)));
                if (claimed) {
                    disc |= 1u << j;
                    p.labels[v[j]] = MP ? u : label;
                }
                ln[j] = claimed ? r1 - st[j] : 0;
                dm += unsigned(ln[j]);
            }
            dn += unsigned(__popc(disc));
            const unsigned enq = disc & ~place4<THREADS>(p, label, disc, st, ln, v, c);
            unsigned total = 0, pre[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const unsigned b = __ballot_sync(FULL, (enq >> j) & 1u);
                pre[j] = total + __popc(b & lt);
                total += __popc(b);
            }
            if (total == 0u) continue;  // warp-uniform
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(qlen_out, total);
            base = __shfl_sync(FULL, base, 0);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if ((enq >> j) & 1u) {
                    const unsigned long long pos = (unsigned long long)base + pre[j];
                    if (pos < (unsigned long long)p.qcap) q_out[pos] = v[j];
                    else atomicOr(&c->error, ERR_OVERFLOW);
                }
            }
        }
    }
    if (p.do_alpha) {
        dn = __reduce_add_sync(FULL, dn);
        dm = __reduce_add_sync(FULL, dm);
        if (lane == 0 && dn) {
            atomicAdd(&c->nf[(it + 1) & 3], dn);
            add_mf_low(c, it + 1, dm);
        }
    }
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ec_fused_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    WarpStage *stg = nullptr;  // this warp's bottom-up stage buffers
    unsigned phase = 0;        // parity their mbarriers complete next
    if constexpr (stage_fits<THREADS, MP>()) {
        if (p.stage_bu) {
            extern __shared__ __align__(128) unsigned char dyn_smem[];
            stg = reinterpret_cast<WarpStage *>(dyn_smem + ec_stage_offset<THREADS, MP>()) + (threadIdx.x >> 5);
            if (lane_id() == 0) {
                mbar_init(&stg->bar[0], 1u);
                mbar_init(&stg->bar[1], 1u);
                mbar_init_fence();
            }
            __syncwarp();
        }
    }
    const uint64_t pol = column_policy(p);
    Counters *c = p.ctr;
    DirectionChoice dir;
    BusyClock clk;
    // A narrow launch may have run the first levels: resume after them, with
    // the direction state they handed over.
    int it = __ldcg(&c->resume);
    if (it > 0) dir.load(c);
    const bool dcounts = p.do_alpha != 0u;
    LevelCounts lc = read_counts(c, it, dcounts, sm);
    const bool failed = ld_relaxed_gpu(&c->error) != 0u;  // as ce_search
    for (; !failed;) {
        clk.start(p);
        const unsigned L = lc.L, nch = lc.nch, nw = lc.nw;
        if (stop_level_loop(p, it, L + nch + nw)) break;
        bool bottom_up = false;
        if (p.do_alpha) bottom_up = dir.next(p, lc.nf, lc.mf);
        if (leader()) {
            ring_prepare(c, it);
            atomicAdd(&c->total_queued, (unsigned long long)L);
            log_phase(p, it, L, nch, nw, bottom_up ? 1u : 0u);
        }
        if (bottom_up) {
            if constexpr (MP) {  // predecessor labels: probes read a snapshot of the visited mask
                snapshot_mask(p);
                if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
            }
            const unsigned done = dir.visited + lc.zmarked;
            bu_level<THREADS, MP>(p, it, sm, done < unsigned(p.nodes) ? unsigned(p.nodes) - done : 0u, stg, phase);
        } else {
            ec_level<THREADS, MP>(p, it, L, nch, nw, sm, pol);
        }
        clk.stop(p);
        log_work_end(p, it);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, it + 1, dcounts))) break;
        lc = sm.lc;
        it++;
    }
    clk.flush(p);
    finish_search(p, it, it);
}

// Contract-expand level of a narrow launch (at most a few thousand queued
// edges on one cluster), written for latency: element i of the edge
// frontier goes to lane i % 32 of warp i / 32 (warps numbered across the
// cluster's CTAs); the lane claims its vertex with one atomicOr, the row
// range loaded behind the atomic; lists of warp_th edges and more go to the
// chunk tables (place4: the next level then belongs to the full grid); the
// warp reserves queue room for its other lists with one atomicAdd, and each
// lane copies its own list, the first entries loaded while the reservation
// is in flight.  No history cache, no probe, no staging: a narrow level is a
// chain of round trips, and every step the throughput path adds lengthens it.
// Labels, queue contents (in another order) and counts are ce_level's.
// c: the level counters (the narrow launch's copy in shared memory).
template <int THREADS, bool MP>
__device__ void ce_narrow_level(const BfsParams &p, Counters *c, int it, unsigned L) {
    const int *q_in = p.queue[it & 1];
    const int *pq_in = p.pred_queue[it & 1];
    const int nq = (it + 1) & 1;
    int *q_out = p.queue[nq];
    int *pq_out = p.pred_queue[nq];
    unsigned *qlen_out = &c->qlen[(it + 1) & 3];
    const unsigned W = unsigned(grid_warps());
    const unsigned lane = lane_id();
    unsigned raw = 0;
    for (unsigned w = unsigned(global_warp()); w * 32u < L; w += W) {
        const unsigned i = w * 32u + lane;
        bool ok = i < L;
        const int u = ok ? ld_cg(q_in + i) : 0;
        const int pr = (MP && ok) ? ld_cg(pq_in + i) : 0;
        if (ok && (unsigned)u >= (unsigned)p.nodes) {
            atomicOr(&c->error, ERR_BAD_VERTEX);
            ok = false;
        }
        const unsigned bit = 1u << ((unsigned)u & 31u);
        const unsigned old = ok ? atomicOr(p.mask + ((unsigned)u >> 5), bit) : bit;
        const int r0 = ok ? __ldg(p.row_offsets + u) : 0;  // issued behind the atomic
        const int r1 = ok ? __ldg(p.row_offsets + u + 1) : 0;
        const bool claimed = !(old & bit);
        if (claimed) p.labels[u] = MP ? pr : it;
        const int len = claimed ? r1 - r0 : 0;
        if (p.count_raw) raw += unsigned(len);
        const int st4[4] = {r0, 0, 0, 0}, ln4[4] = {len, 0, 0, 0}, own4[4] = {u, 0, 0, 0};
        const unsigned placed = place4<THREADS>(p, it + 1, len > 0 ? 1u : 0u, st4, ln4, own4, c);
        const int n = placed ? 0 : len;
        const int incl = warp_inclusive_scan(n);
        const unsigned total = (unsigned)__shfl_sync(FULL, incl, 31);
        if (total == 0u) continue;  // warp-uniform
        int first[4];
#pragma unroll
        for (int k = 0; k < 4; k++) first[k] = k < n ? __ldg(p.col + r0 + k) : 0;
        unsigned base = 0;
        if (lane == 31) base = atomicAdd(qlen_out, total);
        base = __shfl_sync(FULL, base, 31);
        const unsigned long long pos = (unsigned long long)base + unsigned(incl - n);
        for (int k = 0; k < n; k++) {
            const int v = k == 0 ? first[0] : k == 1 ? first[1] : k == 2 ? first[2] : k == 3 ? first[3]
                                                                                          : __ldg(p.col + r0 + k);
            if (pos + k < (unsigned long long)p.qcap) {
                q_out[pos + k] = v;
                if (MP) pq_out[pos + k] = u;
            } else {
                atomicOr(&c->error, ERR_OVERFLOW);
            }
        }
    }
    if (p.count_raw) {
        raw = __reduce_add_sync(FULL, raw);
        if (lane == 0 && raw) atomicAdd(&c->raw[(it + 1) & 3], raw);
    }
}

// Contract-expand level on the full grid for levels of at most one queued
// edge per thread (flat_level): ce_narrow_level's latency-first body, with
// element i going to thread i / G of CTA i % G (G = gridDim.x: a small level
// spreads over every SM), in rounds of G x THREADS elements.  One element per
// thread and round: these levels are chains of round trips whose length is
// set by the instructions between them, and a body with 4 elements in flight
// measured slower on every lattice level, the small ones most.  Each CTA
// reserves the queue room of its round with ONE atomicAdd, scanned over its
// warps in shared memory: per-warp reservations would put thousands of
// atomics on the queue length per level.  Labels, queue contents (in another
// order) and counts are ce_level's.
// it: the level (the label of a claimed vertex); q: its ring phase (q == it
// except in the hybrid kernel, whose two-phase levels take two phases).
template <int THREADS, bool MP>
__device__ void ce_flat_level(const BfsParams &p, int it, int q, unsigned L, Smem<THREADS, MP> &sm) {
    constexpr int NW = THREADS / 32;
    Counters *c = p.ctr;
    const int *q_in = p.queue[q & 1];
    const int *pq_in = p.pred_queue[q & 1];
    const int nq = (q + 1) & 1;
    int *q_out = p.queue[nq];
    int *pq_out = p.pred_queue[nq];
    unsigned *qlen_out = &c->qlen[(q + 1) & 3];
    const unsigned warp = threadIdx.x >> 5, lane = lane_id();
    const unsigned long long G = gridDim.x, round = G * THREADS;
    unsigned raw = 0;
    for (unsigned long long r0 = 0; r0 < L; r0 += round) {  // CTA-uniform
        const unsigned long long i = r0 + (unsigned long long)threadIdx.x * G + blockIdx.x;
        bool ok = i < L;
        const int u = ok ? ld_cg(q_in + i) : 0;
        const int pr = (MP && ok) ? ld_cg(pq_in + i) : 0;
        if (ok && (unsigned)u >= (unsigned)p.nodes) {
            atomicOr(&c->error, ERR_BAD_VERTEX);
            ok = false;
        }
        const unsigned bit = 1u << ((unsigned)u & 31u);
        const unsigned old = ok ? atomicOr(p.mask + ((unsigned)u >> 5), bit) : bit;
        const int r0v = ok ? __ldg(p.row_offsets + u) : 0;  // issued behind the atomic
        const int r1v = ok ? __ldg(p.row_offsets + u + 1) : 0;
        const bool claimed = !(old & bit);
        if (claimed) p.labels[u] = MP ? pr : it;
        const int len = claimed ? r1v - r0v : 0;
        if (p.count_raw) raw += unsigned(len);
        const int st4[4] = {r0v, 0, 0, 0}, ln4[4] = {len, 0, 0, 0}, own4[4] = {u, 0, 0, 0};
        const unsigned placed = place4<THREADS>(p, q + 1, len > 0 ? 1u : 0u, st4, ln4, own4);
        const int n = placed ? 0 : len;
        int first[4];
#pragma unroll
        for (int k = 0; k < 4; k++) first[k] = k < n ? __ldg(p.col + r0v + k) : 0;
        const int incl = warp_inclusive_scan(n);
        if (lane == 31) sm.w[warp].gofs[0] = incl;  // the warp's total
        __syncthreads();
        if (warp == 0) {
            const int t = lane < unsigned(NW) ? sm.w[lane].gofs[0] : 0;
            const int winc = warp_inclusive_scan(t);
            const unsigned total = (unsigned)__shfl_sync(FULL, winc, 31);
            unsigned base = 0;
            if (lane == 0 && total) base = atomicAdd(qlen_out, total);
            base = __shfl_sync(FULL, base, 0);
            if (lane < unsigned(NW)) sm.w[lane].gofs[1] = int(base + unsigned(winc - t));
        }
        __syncthreads();
        // (the next round writes gofs[0] only after every warp has read gofs[1]:
        // its first __syncthreads waits for them)
        const unsigned long long pos = (unsigned long long)(unsigned)sm.w[warp].gofs[1] + unsigned(incl - n);
        for (int k = 0; k < n; k++) {
            const int v = k == 0 ? first[0] : k == 1 ? first[1] : k == 2 ? first[2] : k == 3 ? first[3]
                                                                                          : __ldg(p.col + r0v + k);
            if (pos + k < (unsigned long long)p.qcap) {
                q_out[pos + k] = v;
                if (MP) pq_out[pos + k] = u;
            } else {
                atomicOr(&c->error, ERR_OVERFLOW);
            }
        }
    }
    if (p.count_raw) {
        raw = __reduce_add_sync(FULL, raw);
        if (lane == 0 && raw) atomicAdd(&c->raw[(q + 1) & 3], raw);
    }
}

// Whether a full-grid contract-expand level runs ce_flat_level: no chunked
// lists, at most p.flat_max queued edges, and at most one per grid thread.
// A second round of the latency-first body costs more than the tiled body
// saves (grid3d 256^3: 4.72 ms with levels up to one round, 4.91 ms with
// levels up to 262,144 edges, 1.7 rounds, on a 296 x 512 grid).
template <int THREADS>
__device__ __forceinline__ bool flat_level(const BfsParams &p, unsigned L, unsigned chunks) {
    return chunks == 0u && L <= p.flat_max && L <= gridDim.x * unsigned(THREADS);
}

// The contract-expand level loop of the full grid.  It starts at
// Counters::resume: 0, or the first level a narrow launch before it left.
template <int THREADS, bool MP>
__device__ __forceinline__ void ce_search(const BfsParams &p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const uint64_t pol = column_policy(p);
    Counters *c = p.ctr;
    BusyClock clk;
    int it = __ldcg(&c->resume);
    LevelCounts lc = read_counts(c, it, false, sm);
    // A narrow launch before this one raised an error: no level runs.  (A CTA
    // may also see an error another CTA raised in its first level and leave
    // at once; the others' grid barrier ends on the error.)
    const bool failed = ld_relaxed_gpu(&c->error) != 0u;
    for (; !failed;) {
        clk.start(p);
        const unsigned L = lc.L, nch = lc.nch, nw = lc.nw;
        // raw: the edge frontier before the gather-time cull, so the loop runs
        // (and counts) the levels the reference runs, the last one empty here
        if (stop_level_loop(p, it, L + nch + nw + lc.raw)) break;
        if (leader()) {
            ring_prepare(c, it);
            atomicAdd(&c->total_queued, (unsigned long long)lc.raw);
            log_phase(p, it, lc.raw ? lc.raw : L, nch, nw);
        }
        if (flat_level<THREADS>(p, L, nch + nw))
            ce_flat_level<THREADS, MP>(p, it, it, L, sm);
        else
            ce_level<THREADS, MP>(p, it, it, L, nch, nw, sm, pol);
        clk.stop(p);
        log_work_end(p, it);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, it + 1, false))) break;
        lc = sm.lc;
        it++;
    }
    clk.flush(p);
    finish_search(p, it, it);
}

// A level's counts from counters in shared memory (a narrow launch's); dir:
// also the direction switch's counts.
__device__ __forceinline__ LevelCounts shared_counts(const Counters *c, int q, bool dir = false) {
    const volatile Counters *v = c;
    LevelCounts r{};
    r.L = v->qlen[q & 3];
    r.nch = v->big[q & 3];
    r.nw = v->wch[q & 3];
    r.raw = v->raw[q & 3];
    if (dir) {
        r.nf = v->nf[q & 3];
        r.mf = v->mf[q & 3];
    }
    return r;
}

// The contract-expand level loop of a narrow launch: ONE thread-block
// cluster (gridDim.x CTAs: the helpers spread work over gridDim, so it is
// the grid) runs the search's first levels with ce_narrow_level while their
// input is at most p.narrow_max queued edges without chunked lists, and
// leaves the first larger level to the full-grid launch after it
// (Counters::resume).  A level of a high-diameter graph is a few thousand
// edges; on the full grid its time is mostly latency: the grid barrier, the
// counts read back from L2 after it, the queue reservation's L2 atomic.
// Here the levels end at the cluster's hardware barrier, and the per-level
// counters live in CTA 0's shared memory, which every CTA of the cluster
// reaches as distributed shared memory: reservations and count reads are
// shared-memory round trips.  CTA 0 copies the counters in from global memory
// at the start and the ring entries and error bits back at the end (the
// total_queued sum stays in global memory).  Every CTA leaves the loop on the
// same counts, read after the same barrier, never on the error word: the
// hardware barrier has no timeout, and a CTA missing from it would stall the
// others.
template <int THREADS, bool MP>
__device__ __forceinline__ void ce_narrow_search(const BfsParams &p) {
    __shared__ Counters shared_ctr;  // CTA 0's copy serves the cluster
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    Counters *g = p.ctr;
    constexpr int WORDS = int(offsetof(Counters, sticky) / 4);
    if (blockIdx.x == 0) {
        const unsigned *from = reinterpret_cast<const unsigned *>(g);
        unsigned *to = reinterpret_cast<unsigned *>(&shared_ctr);
        for (int i = threadIdx.x; i < WORDS; i += THREADS) to[i] = __ldcg(from + i);
    }
    cluster_sync_all();
    Counters *c = cooperative_groups::this_cluster().map_shared_rank(&shared_ctr, 0);
    int it = __ldcg(&g->resume);
    if (threadIdx.x == 0) sm.lc = shared_counts(c, it);
    __syncthreads();
    LevelCounts lc = sm.lc;
    for (;;) {
        const unsigned L = lc.L, nch = lc.nch, nw = lc.nw;
        if (L + nch + nw + lc.raw == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (leader()) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        // hand over levels with chunked lists, levels above the bound, and a
        // queue that overflowed (its entries beyond qcap were never written;
        // the full-grid launch sees the error and stops)
        if (nch + nw != 0u || L > p.narrow_max || (long long)L > p.qcap) break;
        if (leader()) {
            ring_prepare(c, it);
            atomicAdd(&g->total_queued, (unsigned long long)lc.raw);
            log_phase(p, it, lc.raw ? lc.raw : L, nch, nw);
        }
        ce_narrow_level<THREADS, MP>(p, c, it, L);
        log_work_end(p, it);
        cluster_sync_all();
        if (threadIdx.x == 0) sm.lc = shared_counts(c, it + 1);
        __syncthreads();
        lc = sm.lc;
        it++;
    }
    cluster_sync_all();  // no CTA touches CTA 0's counters after this
    if (blockIdx.x == 0 && threadIdx.x < 4) {
        const int k = threadIdx.x;
        g->qlen[k] = shared_ctr.qlen[k];
        g->steal[k] = shared_ctr.steal[k];
        g->big[k] = shared_ctr.big[k];
        g->wch[k] = shared_ctr.wch[k];
        g->raw[k] = shared_ctr.raw[k];
        if (k == 0) {
            if (shared_ctr.error) atomicOr(&g->error, shared_ctr.error);
            g->resume = it;  // the full-grid launch ends the search (or finds it ended)
        }
    }
}

// The expand-contract level loop of a narrow launch: ce_narrow_search's
// structure (one cluster, counters in CTA 0's shared memory, levels ending at
// the cluster's hardware barrier) around ec_narrow_level.  With the
// direction switch on, each level's direction is decided as the full-grid
// kernel decides it, on a copy of the state: the first level that would run
// bottom-up goes to the full grid, with the state as it was before that
// level (Counters::dir_*), so the full-grid kernel takes the same decisions.
template <int THREADS, bool MP>
__device__ __forceinline__ void ec_narrow_search(const BfsParams &p) {
    __shared__ Counters shared_ctr;  // CTA 0's copy serves the cluster
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    Counters *g = p.ctr;
    constexpr int WORDS = int(offsetof(Counters, sticky) / 4);
    if (blockIdx.x == 0) {
        const unsigned *from = reinterpret_cast<const unsigned *>(g);
        unsigned *to = reinterpret_cast<unsigned *>(&shared_ctr);
        for (int i = threadIdx.x; i < WORDS; i += THREADS) to[i] = __ldcg(from + i);
    }
    cluster_sync_all();
    Counters *c = cooperative_groups::this_cluster().map_shared_rank(&shared_ctr, 0);
    const bool dcounts = p.do_alpha != 0u;
    DirectionChoice dir;  // a search's state before its level 0
    int it = __ldcg(&g->resume);
    if (threadIdx.x == 0) sm.lc = shared_counts(c, it, dcounts);
    __syncthreads();
    LevelCounts lc = sm.lc;
    for (;;) {
        const unsigned L = lc.L, nch = lc.nch, nw = lc.nw;
        if (L + nch + nw == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (leader()) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        if (nch + nw != 0u || L > p.narrow_max || (long long)L > p.qcap) break;
        if (dcounts) {
            DirectionChoice next = dir;
            if (next.next(p, lc.nf, lc.mf)) break;  // bottom-up: the full grid's level
            dir = next;
        }
        if (leader()) {
            ring_prepare(c, it);
            atomicAdd(&g->total_queued, (unsigned long long)L);
            log_phase(p, it, L, nch, nw, 0u);
        }
        ec_narrow_level<THREADS, MP>(p, c, it, L);
        log_work_end(p, it);
        cluster_sync_all();
        if (threadIdx.x == 0) sm.lc = shared_counts(c, it + 1, dcounts);
        __syncthreads();
        lc = sm.lc;
        it++;
    }
    cluster_sync_all();  // no CTA touches CTA 0's counters after this
    if (blockIdx.x == 0 && threadIdx.x < 4) {
        const int k = threadIdx.x;
        g->qlen[k] = shared_ctr.qlen[k];
        g->steal[k] = shared_ctr.steal[k];
        g->big[k] = shared_ctr.big[k];
        g->wch[k] = shared_ctr.wch[k];
        g->raw[k] = shared_ctr.raw[k];
        g->nf[k] = shared_ctr.nf[k];
        g->mf[k] = shared_ctr.mf[k];
        if (k == 0) {
            if (shared_ctr.error) atomicOr(&g->error, shared_ctr.error);
            dir.store(g);
            g->resume = it;
        }
    }
}

// Expand-contract levels of small frontiers on one thread-block cluster,
// launched before ec_fused_kernel.
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ec_narrow_kernel(BfsParams p) {
    ec_narrow_search<THREADS, MP>(p);
}

// Two-phase contract phase qi = 2 * it of a narrow launch (latency first, as
// ce_narrow_level): element i of the edge frontier goes to lane i % 32 of warp
// i / 32; the lane claims its vertex with one atomicOr, labels it it, and the
// warp appends the claimed vertices to the vertex queue with one atomicAdd.
// c: the level counters (the narrow launch's copy in shared memory).
template <int THREADS, bool MP>
__device__ void tp_narrow_contract(const BfsParams &p, Counters *c, int it, int qi, unsigned L) {
    const int *q_in = p.queue[qi & 1];
    const int *pq_in = p.pred_queue[qi & 1];
    int *q_out = p.queue[(qi + 1) & 1];
    unsigned *qlen_out = &c->qlen[(qi + 1) & 3];
    const unsigned W = unsigned(grid_warps()), lane = lane_id(), lt = lanemask_lt();
    for (unsigned w = unsigned(global_warp()); w * 32u < L; w += W) {
        const unsigned i = w * 32u + lane;
        bool ok = i < L;
        const int u = ok ? ld_cg(q_in + i) : 0;
        const int pr = (MP && ok) ? ld_cg(pq_in + i) : 0;
        if (ok && (unsigned)u >= (unsigned)p.nodes) {
            atomicOr(&c->error, ERR_BAD_VERTEX);
            ok = false;
        }
        const unsigned bit = 1u << ((unsigned)u & 31u);
        const bool claimed = ok && !(atomicOr(p.mask + ((unsigned)u >> 5), bit) & bit);
        if (claimed) p.labels[u] = MP ? pr : it;
        const unsigned b = __ballot_sync(FULL, claimed);
        if (b == 0u) continue;  // warp-uniform
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(qlen_out, unsigned(__popc(b)));
        base = __shfl_sync(FULL, base, 0);
        if (claimed) {
            const unsigned long long pos = (unsigned long long)base + __popc(b & lt);
            if (pos < (unsigned long long)p.qcap) q_out[pos] = u;
            else atomicOr(&c->error, ERR_OVERFLOW);
        }
    }
}

// Two-phase expand phase qi = 2 * it + 1 of a narrow launch: frontier vertex
// i goes to lane i % 32 of warp i / 32; its list goes to the chunk tables
// when long (place4: the next level is then the full grid's), else the warp
// reserves queue room for its lists with one atomicAdd and each lane copies
// its own, the first entries loaded while the reservation is in flight.
template <int THREADS, bool MP>
__device__ void tp_narrow_expand(const BfsParams &p, Counters *c, int qi, unsigned L) {
    const int *q_in = p.queue[qi & 1];
    const int nq = (qi + 1) & 1;
    int *q_out = p.queue[nq];
    int *pq_out = p.pred_queue[nq];
    unsigned *qlen_out = &c->qlen[(qi + 1) & 3];
    const unsigned W = unsigned(grid_warps()), lane = lane_id();
    unsigned raw = 0;
    for (unsigned w = unsigned(global_warp()); w * 32u < L; w += W) {
        const unsigned i = w * 32u + lane;
        const bool ok = i < L;
        const int u = ok ? ld_cg(q_in + i) : 0;
        const int r0 = ok ? __ldg(p.row_offsets + u) : 0;
        const int len = ok ? __ldg(p.row_offsets + u + 1) - r0 : 0;
        if (p.count_raw) raw += unsigned(len);
        const int st4[4] = {r0, 0, 0, 0}, ln4[4] = {len, 0, 0, 0}, own4[4] = {u, 0, 0, 0};
        const unsigned placed = place4<THREADS>(p, qi + 1, len > 0 ? 1u : 0u, st4, ln4, own4, c);
        const int n = placed ? 0 : len;
        const int incl = warp_inclusive_scan(n);
        const unsigned total = (unsigned)__shfl_sync(FULL, incl, 31);
        if (total == 0u) continue;  // warp-uniform
        int first[4];
#pragma unroll
        for (int k = 0; k < 4; k++) first[k] = k < n ? __ldg(p.col + r0 + k) : 0;
        unsigned base = 0;
        if (lane == 31) base = atomicAdd(qlen_out, total);
        base = __shfl_sync(FULL, base, 31);
        const unsigned long long pos = (unsigned long long)base + unsigned(incl - n);
        for (int k = 0; k < n; k++) {
            const int v = k == 0 ? first[0] : k == 1 ? first[1] : k == 2 ? first[2] : k == 3 ? first[3]
                                                                                          : __ldg(p.col + r0 + k);
            if (pos + k < (unsigned long long)p.qcap) {
                q_out[pos + k] = v;
                if (MP) pq_out[pos + k] = u;
            } else {
                atomicOr(&c->error, ERR_OVERFLOW);
            }
        }
    }
    if (p.count_raw) {
        raw = __reduce_add_sync(FULL, raw);
        if (lane == 0 && raw) atomicAdd(&c->raw[(qi + 1) & 3], raw);
    }
}

// The two-phase level loop of a narrow launch: ce_narrow_search's structure
// with both phases of a level on the cluster, each ending at the cluster's
// hardware barrier.  It hands over only before a contract phase (the full-grid
// kernel resumes at phase 2 * Counters::resume).  A contract phase that
// discovers nothing ends the search as the reference does (no ++): the narrow
// launch then finishes it itself (iteration, end marker, sticky error) and sets
// Counters::resume to -1, so the full-grid launch after it does nothing.
template <int THREADS, bool MP>
__device__ __forceinline__ void tp_narrow_search(const BfsParams &p) {
    __shared__ Counters shared_ctr;  // CTA 0's copy serves the cluster
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    Counters *g = p.ctr;
    constexpr int WORDS = int(offsetof(Counters, sticky) / 4);
    if (blockIdx.x == 0) {
        const unsigned *from = reinterpret_cast<const unsigned *>(g);
        unsigned *to = reinterpret_cast<unsigned *>(&shared_ctr);
        for (int i = threadIdx.x; i < WORDS; i += THREADS) to[i] = __ldcg(from + i);
    }
    cluster_sync_all();
    Counters *c = cooperative_groups::this_cluster().map_shared_rank(&shared_ctr, 0);
    int it = __ldcg(&g->resume), qi = 2 * it;
    bool ended = false;  // a contract phase discovered nothing
    if (threadIdx.x == 0) sm.lc = shared_counts(c, qi);
    __syncthreads();
    LevelCounts lc = sm.lc;
    for (;;) {
        const unsigned L = lc.L, nch = lc.nch, nw = lc.nw;
        if (L + nch + nw + lc.raw == 0u) break;
        if (level_limit_hit(it, p.nodes)) {
            if (leader()) atomicOr(&c->error, ERR_LEVEL_LIMIT);
            break;
        }
        if (nch + nw != 0u || L > p.narrow_max || (long long)L > p.qcap) break;
        if (leader()) {
            ring_prepare(c, qi);
            atomicAdd(&g->total_queued, (unsigned long long)lc.raw);
            log_phase(p, qi, lc.raw ? lc.raw : L, nch, nw);
        }
        tp_narrow_contract<THREADS, MP>(p, c, it, qi, L);
        log_work_end(p, qi);
        cluster_sync_all();
        if (threadIdx.x == 0) sm.lc = shared_counts(c, qi + 1);
        __syncthreads();
        const unsigned Lv = sm.lc.L;
        if (Lv == 0u || (long long)Lv > p.qcap) {  // no vertex discovered (or the vertex queue overflowed)
            ended = true;
            break;
        }
        if (leader()) {
            ring_prepare(c, qi + 1);
            log_phase(p, qi + 1, Lv, 0u, 0u);
        }
        tp_narrow_expand<THREADS, MP>(p, c, qi + 1, Lv);
        log_work_end(p, qi + 1);
        cluster_sync_all();
        if (threadIdx.x == 0) sm.lc = shared_counts(c, qi + 2);
        __syncthreads();
        lc = sm.lc;
        qi += 2;
        it++;
    }
    cluster_sync_all();  // no CTA touches CTA 0's counters after this
    if (blockIdx.x == 0 && threadIdx.x < 4) {
        const int k = threadIdx.x;
        g->qlen[k] = shared_ctr.qlen[k];
        g->steal[k] = shared_ctr.steal[k];
        g->big[k] = shared_ctr.big[k];
        g->wch[k] = shared_ctr.wch[k];
        g->raw[k] = shared_ctr.raw[k];
        if (k == 0) {
            if (shared_ctr.error) atomicOr(&g->error, shared_ctr.error);
            g->resume = ended ? -1 : it;
        }
    }
    if (ended && leader()) {  // as tp_fused_kernel's finish after an empty contract
        g->iteration = it;
        log_phase(p, qi + 2, 0u, 0u, 0u);  // end-of-search marker
        atomicOr(&g->sticky, shared_ctr.error | __ldcg(&g->error));
    }
}

// Two-phase levels of small frontiers on one thread-block cluster, launched
// before tp_fused_kernel.
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) tp_narrow_kernel(BfsParams p) {
    tp_narrow_search<THREADS, MP>(p);
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ce_fused_kernel(BfsParams p) {
    ce_search<THREADS, MP>(p);
}

// Contract-expand levels of small frontiers on one thread-block cluster,
// launched before ce_fused_kernel.
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ce_narrow_kernel(BfsParams p) {
    ce_narrow_search<THREADS, MP>(p);
}

// Fused two-phase: contract and expand phases alternate across grid barriers
// (the reference's fused two-phase kernel, two_phase/kernel.cuh:60-313, which
// its enactor cannot instantiate, enactor_two_phase.cuh:302).  The level log is
// indexed by phase (2 * iteration for contract, + 1 for expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) tp_fused_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const uint64_t pol = column_policy(p);
    Counters *c = p.ctr;
    BusyClock clk;
    // A narrow launch may have run the first levels (resume), or the whole
    // search (resume -1: nothing left to do).
    const int resume = __ldcg(&c->resume);
    if (resume < 0) return;
    int it = resume, qi = 2 * resume;
    LevelCounts lc = read_counts(c, qi, false, sm);
    const bool failed = ld_relaxed_gpu(&c->error) != 0u;  // as ce_search
    for (; !failed;) {
        clk.start(p);
        unsigned L = lc.L;
        const unsigned nch = lc.nch, nw = lc.nw;
        if (stop_level_loop(p, it, L + nch + nw + lc.raw)) break;
        const bool cull = gather_cull(level_edges<THREADS>(lc));
        if (leader()) {
            ring_prepare(c, qi);
            atomicAdd(&c->total_queued, (unsigned long long)lc.raw);
            log_phase(p, qi, lc.raw ? lc.raw : L, nch, nw);
        }
        tp_contract<THREADS, MP>(p, it, qi, L, nch, nw, sm, pol);
        clk.stop(p);
        log_work_end(p, qi);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, qi + 1, false))) break;
        clk.start(p);
        qi++;
        L = sm.lc.L;
        if (L == 0u) break;  // no vertex discovered: the reference stops without ++
        if (leader()) {
            ring_prepare(c, qi);
            log_phase(p, qi, L, 0u, 0u);
        }
        tp_expand<THREADS, MP>(p, qi, L, cull, sm, pol);
        clk.stop(p);
        log_work_end(p, qi);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, qi + 1, false))) break;
        lc = sm.lc;
        qi++;
        it++;
    }
    clk.flush(p);
    finish_search(p, it, qi + 1);
}

// Hybrid (the reference's EnactorHybrid, enactor_hybrid.cuh:279-555): a level
// whose incoming edge frontier is small runs as one contract-expand phase; a
// level whose frontier exceeds 4 edges per thread of the grid (the reference's
// SATURATION_QUIT = 4 * 128 per 128-thread CTA, :571, checked by
// contract_expand_atomic/kernel.cuh:653 and two_phase/contract_atomic/kernel.cuh:338)
// runs as a two-phase contract phase and expand phase.  Both bodies take and
// leave the same edge frontier, so the switch happens inside one persistent
// launch instead of between kernels.  Every CTA reads the same counters after
// the barrier and so takes the same branch.  The level log is indexed by phase.
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) hy_fused_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const uint64_t pol = column_policy(p);
    Counters *c = p.ctr;
    const unsigned long long saturation = 4ull * THREADS * gridDim.x;
    BusyClock clk;
    // A narrow launch (contract-expand levels on one cluster, where the ring
    // phase is the level) may have run the first levels.
    int it = __ldcg(&c->resume), q = it;
    LevelCounts lc = read_counts(c, q, false, sm);
    const bool failed = ld_relaxed_gpu(&c->error) != 0u;  // as ce_search
    for (; !failed;) {
        clk.start(p);
        unsigned L = lc.L;
        const unsigned nch = lc.nch, nw = lc.nw;
        if (stop_level_loop(p, it, L + nch + nw + lc.raw)) break;
        if (leader()) {
            ring_prepare(c, q);
            atomicAdd(&c->total_queued, (unsigned long long)lc.raw);
            log_phase(p, q, lc.raw ? lc.raw : L, nch, nw);
        }
        // the level's edge frontier as the reference counts it (before the gather-time cull)
        const unsigned long long edges = level_edges<THREADS>(lc);
        if (edges <= saturation) {
            if (flat_level<THREADS>(p, L, nch + nw))
                ce_flat_level<THREADS, MP>(p, it, q, L, sm);
            else
                ce_level<THREADS, MP>(p, it, q, L, nch, nw, sm, pol);
            clk.stop(p);
            log_work_end(p, q);
            if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, q + 1, false))) break;
            lc = sm.lc;
            q++;
            it++;
            continue;
        }
        const bool cull = gather_cull(edges);
        tp_contract<THREADS, MP>(p, it, q, L, nch, nw, sm, pol);
        clk.stop(p);
        log_work_end(p, q);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, q + 1, false))) break;
        clk.start(p);
        q++;
        L = sm.lc.L;
        if (L == 0u) break;  // no vertex discovered: stop without ++, as two-phase does
        if (leader()) {
            ring_prepare(c, q);
            log_phase(p, q, L, 0u, 0u);
        }
        tp_expand<THREADS, MP>(p, q, L, cull, sm, pol);
        clk.stop(p);
        log_work_end(p, q);
        if (!grid_barrier(c, p.wait_ns, &sm.flag, next_counts(&sm.lc, q + 1, false))) break;
        lc = sm.lc;
        q++;
        it++;
    }
    clk.flush(p);
    finish_search(p, it, q);
}

// ---- per-level kernels for the graph-driven (iterative) variants ----------------

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ec_level_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3], nch = p.ctr->big[it & 3], nw = p.ctr->wch[it & 3];
    if (L + nch + nw == 0u || p.ctr->error) return;
    if (leader()) log_phase(p, it, L, nch, nw);
    ec_level<THREADS, MP>(p, it, L, nch, nw, sm, column_policy(p));
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) ce_level_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it;
    const unsigned L = p.ctr->qlen[it & 3], nch = p.ctr->big[it & 3], nw = p.ctr->wch[it & 3];
    const unsigned raw = p.ctr->raw[it & 3];
    if (L + nch + nw + raw == 0u || p.ctr->error) return;
    if (leader()) log_phase(p, it, raw ? raw : L, nch, nw);
    ce_level<THREADS, MP>(p, it, it, L, nch, nw, sm, column_policy(p));
}

// Two-phase per-level: qi = 2 * it (contract) and 2 * it + 1 (expand).
template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) tp_contract_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it;
    const unsigned L = p.ctr->qlen[qi & 3], nch = p.ctr->big[qi & 3], nw = p.ctr->wch[qi & 3];
    const unsigned raw = p.ctr->raw[qi & 3];
    if (L + nch + nw + raw == 0u || p.ctr->error) return;
    if (leader()) log_phase(p, qi, raw ? raw : L, nch, nw);
    tp_contract<THREADS, MP>(p, it, qi, L, nch, nw, sm, column_policy(p));
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS(THREADS)) tp_expand_kernel(BfsParams p) {
    Smem<THREADS, MP> &sm = kernel_smem<THREADS, MP>();
    init_hist(sm, p.cull_flags);
    const int it = p.ctr->cur_it, qi = 2 * it + 1;
    const unsigned L = p.ctr->qlen[qi & 3];
    if (L == 0u || p.ctr->error) return;
    if (leader()) log_phase(p, qi, L, 0u, 0u);
    const int qc = qi - 1;  // the level's contract phase
    LevelCounts in{};
    in.L = p.ctr->qlen[qc & 3];
    in.nch = p.ctr->big[qc & 3];
    in.nw = p.ctr->wch[qc & 3];
    in.raw = p.ctr->raw[qc & 3];
    tp_expand<THREADS, MP>(p, qi, L, gather_cull(level_edges<THREADS>(in)), sm, column_policy(p));
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
        const unsigned eq =                          // expand output, before and after the gather-time cull
            c->raw[(qi + 2) & 3] + c->qlen[(qi + 2) & 3] + c->big[(qi + 2) & 3] + c->wch[(qi + 2) & 3];
        c->total_queued += c->raw[qi & 3];
        if (vq == 0u) {
            c->iteration = it;  // the reference leaves after contract without ++
            more = false;
        } else {
            c->iteration = it + 1;
            more = eq != 0u;
        }
        // the next body runs phases qi+2 (contract) and qi+3 (expand)
        c->steal[(qi + 2) & 3] = 0u;
        c->steal[(qi + 3) & 3] = 0u;
        c->qlen[(qi + 3) & 3] = 0u;
        c->qlen[(qi + 4) & 3] = 0u;
        c->big[(qi + 3) & 3] = 0u;
        c->big[(qi + 4) & 3] = 0u;
        c->wch[(qi + 3) & 3] = 0u;
        c->wch[(qi + 4) & 3] = 0u;
        c->raw[(qi + 3) & 3] = 0u;
        c->raw[(qi + 4) & 3] = 0u;
        if (!more) log_phase(p, vq == 0u ? qi + 1 : qi + 2, 0u, 0u, 0u);
    } else {
        const bool edge = strategy != STRATEGY_EXPAND_CONTRACT;
        const unsigned next = c->qlen[(it + 1) & 3] + c->big[(it + 1) & 3] + c->wch[(it + 1) & 3] +
                              (edge ? c->raw[(it + 1) & 3] : 0u);
        c->total_queued += edge ? c->raw[it & 3] : c->qlen[it & 3];
        c->iteration = it + 1;
        more = next != 0u;
        c->steal[(it + 1) & 3] = 0u;
        c->qlen[(it + 2) & 3] = 0u;
        c->big[(it + 2) & 3] = 0u;
        c->wch[(it + 2) & 3] = 0u;
        c->raw[(it + 2) & 3] = 0u;
        if (!more) log_phase(p, it + 1, 0u, 0u, 0u);
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

// SplitMix64's output function (Steele, Lea and Flood, OOPSLA 2014) as a 64-bit mixer.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// sums[0] / sums[1]: hash sums of (u, v) / (v, u) over every entry v of row u;
// sums[2] / sums[3]: the same with a second, salted hash.  The entries are cut
// into runs of SYM_RUN consecutive ones, one run per lane (a warp takes 32
// runs): the lane finds the row of its first entry by binary search over the
// row offsets and walks forward from there, so a hub's list is spread over as
// many lanes as it has runs, whatever the vertex order.
constexpr int SYM_RUN = 64;

__device__ __forceinline__ void hash_entry(unsigned u, unsigned v, unsigned long long (&h)[4]) {
    constexpr unsigned long long SALT = 0x5851f42d4c957f2dull;
    const unsigned long long fwd = ((unsigned long long)u << 32) | v;
    const unsigned long long rev = ((unsigned long long)v << 32) | u;
    h[0] += mix64(fwd);
    h[1] += mix64(rev);
    h[2] += mix64(fwd ^ SALT);
    h[3] += mix64(rev ^ SALT);
}

__global__ void symmetry_hash_kernel(const int *row_offsets, const int *col, int nodes, long long edges,
                                     unsigned long long *sums) {
    unsigned long long h[4] = {0, 0, 0, 0};
    const long long W = grid_warps();
    for (long long c = global_warp(); c * 32 * SYM_RUN < edges; c += W) {
        const long long k0 = (c * 32 + lane_id()) * SYM_RUN;
        if (k0 < edges) {
            const long long k1 = min(edges, k0 + SYM_RUN);
            int lo = 0, hi = nodes;  // last row lo with row_offsets[lo] <= k0
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(row_offsets + mid) <= k0) lo = mid;
                else hi = mid;
            }
            int r = lo;
            long long next = __ldg(row_offsets + r + 1);
            for (long long k = k0; k < k1; k++) {
                while (k >= next) next = __ldg(row_offsets + (++r) + 1);
                hash_entry(unsigned(r), (unsigned)__ldg(col + k), h);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) h[j] = (unsigned long long)warp_sum_ll((long long)h[j]);
    if (lane_id() == 0)
#pragma unroll
        for (int j = 0; j < 4; j++) atomicAdd(sums + j, h[j]);
}

// keys[v] = the largest (deg(u) << 32) | u over the entries u of row v: its
// neighbour of highest degree, which bottom-up levels probe before reading the
// list (the highest-degree vertices are reached first, so on graphs with a
// skewed degree distribution that one neighbour is nearly always the parent
// when there is one).  Runs of HEAVY_RUN entries per lane, found and walked
// as in the symmetry check; a lane folds each row's best key into keys[row]
// with one atomicMax per row it touches, so a hub's list costs one atomic per
// run.  Out-of-range entries are skipped (the CSR check rejects them first).
constexpr int HEAVY_RUN = 64;

__global__ void heavy_neighbour_kernel(const int *row_offsets, const int *col, int nodes, long long edges,
                                       unsigned long long *keys) {
    const long long W = grid_warps();
    for (long long c = global_warp(); c * 32 * HEAVY_RUN < edges; c += W) {
        const long long k0 = (c * 32 + lane_id()) * HEAVY_RUN;
        if (k0 >= edges) continue;
        const long long k1 = min(edges, k0 + HEAVY_RUN);
        int lo = 0, hi = nodes;  // last row lo with row_offsets[lo] <= k0
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(row_offsets + mid) <= k0) lo = mid;
            else hi = mid;
        }
        int r = lo;
        long long next = __ldg(row_offsets + r + 1);
        unsigned long long best = 0;
        for (long long k = k0; k < k1; k += 4) {
            int u[4], d0[4], d1[4];
#pragma unroll
            for (int j = 0; j < 4; j++) u[j] = k + j < k1 ? __ldg(col + k + j) : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int uu = (unsigned)u[j] < (unsigned)nodes ? u[j] : 0;
                d0[j] = __ldg(row_offsets + uu);
                d1[j] = __ldg(row_offsets + uu + 1);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (k + j >= k1) break;
                while (k + j >= next) {  // entry k + j belongs to a later row
                    if (best) atomicMax(keys + r, best);
                    best = 0;
                    next = __ldg(row_offsets + (++r) + 1);
                }
                if ((unsigned)u[j] < (unsigned)nodes) {
                    const unsigned long long key =
                        ((unsigned long long)(unsigned)(d1[j] - d0[j]) << 32) | (unsigned)u[j];
                    best = key > best ? key : best;
                }
            }
        }
        if (best) atomicMax(keys + r, best);
    }
}

// Reset's initialisation in one launch: labels := -1 (16-byte stores; the
// array is cudaMalloc-aligned) and the visited mask := 0.
__global__ void reset_state_kernel(int *labels, long long n, unsigned *mask, long long mask_words) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n4 = n >> 2;
    int4 *l4 = reinterpret_cast<int4 *>(labels);
    for (long long i = t; i < n4; i += stride) l4[i] = make_int4(-1, -1, -1, -1);
    for (long long i = (n4 << 2) + t; i < n; i += stride) labels[i] = -1;
    for (long long i = t; i < mask_words; i += stride) mask[i] = 0u;
}

// CSR checks on the device: out[0] = the first row v whose offsets decrease
// (row[v+1] < row[v]), out[1] = the first entry outside [0, nodes); both stay
// ~0 when there is none (out must start at ~0).
__global__ void csr_check_kernel(const int *row_offsets, const int *col, int nodes, long long edges,
                                 unsigned long long *out) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long v = t; v < nodes; v += stride)
        if (__ldg(row_offsets + v + 1) < __ldg(row_offsets + v)) atomicMin(out + 0, (unsigned long long)v);
    for (long long k = t; k < edges; k += stride)
        if ((unsigned)__ldg(col + k) >= (unsigned)nodes) atomicMin(out + 1, (unsigned long long)k);
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
    case STRATEGY_HYBRID: return hy_fused_kernel<THREADS, MP>;
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

template <bool MP>
static size_t smem_bytes_t(int threads) {
    switch (threads) {
    case 128: return sizeof(Smem<128, MP>);
    case 512: return sizeof(Smem<512, MP>);
    default: return sizeof(Smem<256, MP>);
    }
}

static size_t smem_bytes(const KernelConfig &kc) {
    return kc.mark_pred ? smem_bytes_t<true>(kc.threads) : smem_bytes_t<false>(kc.threads);
}

// The fused kernels' dynamic shared memory: the expand-contract kernel adds
// its bottom-up stage buffers where they fit.
template <bool MP>
static size_t fused_smem_bytes_t(int threads, int strategy) {
    if (strategy != STRATEGY_EXPAND_CONTRACT) return smem_bytes_t<MP>(threads);
    switch (threads) {
    case 128: return ec_smem_bytes<128, MP>();
    case 512: return ec_smem_bytes<512, MP>();
    default: return ec_smem_bytes<256, MP>();
    }
}
static size_t fused_smem_bytes(const KernelConfig &kc) {
    if (!kc.stage_bu) return smem_bytes(kc);  // the stage buffers take L1 capacity: only when used
    return kc.mark_pred ? fused_smem_bytes_t<true>(kc.threads, kc.strategy)
                        : fused_smem_bytes_t<false>(kc.threads, kc.strategy);
}

// Opts a kernel in to its dynamic shared memory size (beyond 48 KB needs it).
static cudaError_t allow_smem(const void *fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

static KernelFn pick_fused(const KernelConfig &kc) {
    return kc.mark_pred ? fused_fn_t<true>(kc.threads, kc.strategy) : fused_fn_t<false>(kc.threads, kc.strategy);
}

// The hybrid's first levels are contract-expand levels: the same narrow kernel
// runs them, and hy_fused_kernel resumes after it.  Expand-contract has its own.
template <bool MP>
static KernelFn narrow_fn_t(int threads, int strategy) {
    if (strategy == STRATEGY_TWO_PHASE) {
        switch (threads) {
        case 128: return tp_narrow_kernel<128, MP>;
        case 512: return tp_narrow_kernel<512, MP>;
        default: return tp_narrow_kernel<256, MP>;
        }
    }
    if (strategy == STRATEGY_EXPAND_CONTRACT) {
        switch (threads) {
        case 128: return ec_narrow_kernel<128, MP>;
        case 512: return ec_narrow_kernel<512, MP>;
        default: return ec_narrow_kernel<256, MP>;
        }
    }
    switch (threads) {  // contract-expand, hybrid
    case 128: return ce_narrow_kernel<128, MP>;
    case 512: return ce_narrow_kernel<512, MP>;
    default: return ce_narrow_kernel<256, MP>;
    }
}
static KernelFn pick_narrow(const KernelConfig &kc) {
    return kc.mark_pred ? narrow_fn_t<true>(kc.threads, kc.strategy) : narrow_fn_t<false>(kc.threads, kc.strategy);
}

static cudaLaunchConfig_t narrow_config(const KernelConfig &kc, int team, cudaStream_t stream,
                                        cudaLaunchAttribute *attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(team));
    cfg.blockDim = dim3(unsigned(kc.threads));
    cfg.dynamicSmemBytes = fused_smem_bytes(kc);
    cfg.stream = stream;
    attr->id = cudaLaunchAttributeClusterDimension;
    attr->val.clusterDim.x = unsigned(team);
    attr->val.clusterDim.y = 1;
    attr->val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

cudaError_t narrow_team_limit(const KernelConfig &kc, int want, int *team) {
    *team = 0;
    KernelFn fn = pick_narrow(kc);
    if (!fn || want < 1) return cudaSuccess;
    cudaError_t e = allow_smem((const void *)fn, fused_smem_bytes(kc));
    if (e) return e;
    if ((e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
    for (int t = std::min(want, 16); t >= 1; t--) {
        cudaLaunchAttribute attr;
        cudaLaunchConfig_t cfg = narrow_config(kc, t, nullptr, &attr);
        int clusters = 0;
        if ((e = cudaOccupancyMaxActiveClusters(&clusters, (const void *)fn, &cfg))) {
            cudaGetLastError();  // a size the device refuses: try a smaller one
            continue;
        }
        if (clusters >= 1) {
            *team = t;
            return cudaSuccess;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_narrow(const BfsParams &p, const KernelConfig &kc, int team, cudaStream_t stream) {
    KernelFn fn = pick_narrow(kc);
    if (!fn || team < 1 || team > 16) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t cfg = narrow_config(kc, team, stream, &attr);
    BfsParams arg = p;
    return cudaLaunchKernelEx(&cfg, fn, arg);
}

struct LevelFns {
    KernelFn level_a;  // ec_level / ce_level / tp_contract
    KernelFn level_b;  // tp_expand for two-phase
};

template <int THREADS, bool MP>
static LevelFns level_fns(int strategy) {
    LevelFns f{};
    switch (strategy) {
    case STRATEGY_EXPAND_CONTRACT: f.level_a = ec_level_kernel<THREADS, MP>; break;
    case STRATEGY_CONTRACT_EXPAND: f.level_a = ce_level_kernel<THREADS, MP>; break;
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

static cudaError_t grid_for(const void *fn, int threads, size_t smem, int *grid) {
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    if ((e = allow_smem(fn, smem))) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem);
    if (e) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    *grid = sms * occ;
    return cudaSuccess;
}

cudaError_t launch_search_init(const BfsParams &p, const KernelConfig &kc, cudaStream_t stream) {
    const int cta_chunk = kc.threads == 128 ? chunk_edges<128>() : kc.threads == 512 ? chunk_edges<512>()
                                                                                       : chunk_edges<256>();
    search_init_kernel<<<1, 64, 0, stream>>>(p, kc.strategy, kc.mark_pred ? 1 : 0, cta_chunk);
    return cudaGetLastError();
}

cudaError_t fused_grid_limit(const KernelConfig &kc, int *grid) {
    return grid_for((const void *)pick_fused(kc), kc.threads, fused_smem_bytes(kc), grid);
}

cudaError_t level_grid_limit(const KernelConfig &kc, int *grid) {
    LevelFns f = pick_level(kc);
    if (f.level_b) {
        cudaError_t e = allow_smem((const void *)f.level_b, smem_bytes(kc));
        if (e) return e;
    }
    return grid_for((const void *)f.level_a, kc.threads, smem_bytes(kc), grid);
}

cudaError_t launch_symmetry_hash(const int *row_offsets, const int *col, int nodes, long long edges,
                                 unsigned long long *sums, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    symmetry_hash_kernel<<<sms * 8, 256, 0, stream>>>(row_offsets, col, nodes, edges, sums);
    return cudaGetLastError();
}

cudaError_t launch_heavy_neighbour(const int *row_offsets, const int *col, int nodes, long long edges,
                                   unsigned long long *keys, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    heavy_neighbour_kernel<<<sms * 8, 256, 0, stream>>>(row_offsets, col, nodes, edges, keys);
    return cudaGetLastError();
}

cudaError_t launch_reset_state(int *labels, long long nodes, unsigned *mask, long long mask_words,
                               cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    reset_state_kernel<<<sms * 8, 256, 0, stream>>>(labels, nodes, mask, mask_words);
    return cudaGetLastError();
}

cudaError_t launch_csr_check(const int *row_offsets, const int *col, int nodes, long long edges,
                             unsigned long long *out, cudaStream_t stream) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e) return e;
    csr_check_kernel<<<sms * 8, 256, 0, stream>>>(row_offsets, col, nodes, edges, out);
    return cudaGetLastError();
}

cudaError_t launch_fused(const BfsParams &p, const KernelConfig &kc, int grid, cudaStream_t stream) {
    KernelFn fn = pick_fused(kc);
    const size_t smem = fused_smem_bytes(kc);
    cudaError_t e = allow_smem((const void *)fn, smem);
    if (e) return e;
    BfsParams arg = p;
    void *args[] = {&arg};
    return cudaLaunchCooperativeKernel((const void *)fn, dim3(grid), dim3(kc.threads), args, smem, stream);
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
        const size_t smem = smem_bytes(kc);
        if ((e = allow_smem((const void *)f.level_a, smem))) break;
        if (f.level_b && (e = allow_smem((const void *)f.level_b, smem))) break;
        f.level_a<<<grid, T, smem, cap>>>(p);
        if (f.level_b) f.level_b<<<grid, T, smem, cap>>>(p);
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
