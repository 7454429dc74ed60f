// Multi-search BFS kernels (sm_100a): many searches over many resident graphs
// advance together in one persistent cooperative launch.
//
// The batch runs the expand-contract strategy of bfs_kernels.cu with every
// work item tagged by its search slot: frontier entries are (slot, vertex)
// pairs and grid-wide chunk descriptors carry the slot in their last field.
// Each slot has its own labels and visited mask (offsets into shared pools)
// and its graph (an entry of the resident-graph table).  All slots share one
// grid barrier per level, so small searches ride along with large ones instead
// of paying a launch and a level loop each -- the point of batching.
//
// Slots may start at different levels (the serving loop admits new searches
// between launches): a search's depth labels count from its start level.  At
// the start of every level one CTA retires the slots that received no input
// for it, recording the iteration count and %globaltimer of completion.

#include <cuda_runtime.h>

#include <cstddef>

#include "ms_kernels.cuh"

namespace b40c_b200 {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WINDOW = 128;
constexpr int OBUF = 256;

#define MS_MIN_BLOCKS(threads) (1024 / (threads))

template <bool MP>
struct MsWarp {
    const int *gaddr[WINDOW];  // scan-gather window: address of each column entry
    int gslot[WINDOW];
    int gpred[MP ? WINDOW : 1];
    int2 obuf[OBUF];           // staged (slot, vertex) appends
    unsigned nbuf;
};

template <int THREADS, bool MP>
struct MsSmem {
    MsWarp<MP> w[THREADS / 32];
    unsigned long long vcache[VCACHE];  // (global mask word << 32) | word value
    unsigned warp_tot[THREADS / 32];    // bookkeeping scan of bottom-up steps
    LevelCounts lc;                     // a level's counts, read once per CTA
    unsigned flag;
    unsigned last;                      // grid_barrier_serial: this CTA arrived last
};

template <int THREADS, bool MP>
__device__ __forceinline__ MsSmem<THREADS, MP> &ms_smem() {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    return *reinterpret_cast<MsSmem<THREADS, MP> *>(dyn_smem);
}

__device__ __forceinline__ bool leader() { return blockIdx.x == 0 && threadIdx.x == 0; }
// Warp w of the grid is warp w / gridDim.x of CTA w % gridDim.x: consecutive
// work items (tiles, steps, runs) go to different CTAs, and so to different
// SMs, so a level with few items still spreads over the whole GPU instead of
// crowding the issue slots and memory pipes of the first few SMs.
__device__ __forceinline__ int global_warp() { return int((threadIdx.x >> 5) * gridDim.x + blockIdx.x); }
__device__ __forceinline__ int grid_warps() { return int(gridDim.x * (blockDim.x >> 5)); }

__device__ __forceinline__ MsSlot load_slot(const MsParams &p, int s) {
    MsSlot d;
    const int4 *q = reinterpret_cast<const int4 *>(p.slots + s);
    int4 a = __ldg(q), b = __ldg(q + 1);
    d.label_off = (long long)(unsigned)a.x | ((long long)a.y << 32);
    d.mask_off = (long long)(unsigned)a.z | ((long long)a.w << 32);
    d.graph = b.x;
    d.start_level = b.y;
    d.nodes = b.z;
    d.pad = b.w;
    return d;
}
static_assert(sizeof(MsSlot) == 32, "load_slot reads two int4");

__device__ __forceinline__ void mark_alive(const MsParams &p, int q, int slot) {
    unsigned char *a = p.alive + size_t(q & 3) * size_t(p.nslots) + slot;
    if (*a == 0) *a = 1;  // a stale 0 only costs a repeated store
}

// ---- placement of discovered lists ---------------------------------------------------

template <int CH>
__device__ __forceinline__ unsigned ms_place_tier(int4 *table, unsigned *count, int cap, unsigned sel, int n,
                                                  const int (&nc)[4], const int (&st)[4], const int (&ln)[4],
                                                  const int (&pr)[4], const int (&sl)[4]) {
    const int incl = warp_inclusive_scan(n);
    const unsigned total = (unsigned)__shfl_sync(FULL, incl, 31);
    if (total == 0u) return 0u;
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
                    table[my++] = make_int4(cs, ce - cs, pr[j], sl[j]);
                }
            }
        }
        return sel;
    }
    for (unsigned c = my; c < (unsigned)cap && c < my + unsigned(n); c++) table[c] = make_int4(0, 0, 0, 0);
    return 0u;
}

template <int THREADS>
__device__ __forceinline__ unsigned ms_place4(const MsParams &p, int q_next, unsigned has, const int (&st)[4],
                                              const int (&ln)[4], const int (&pr)[4], const int (&sl)[4]) {
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
    unsigned placed =
        ms_place_tier<CH>(p.chunks[nq], &p.ctr->big[q_next & 3], p.chunk_cap, cta, ncta, nc, st, ln, pr, sl);
    placed |= ms_place_tier<WARP_CHUNK>(p.wchunks[nq], &p.ctr->wch[q_next & 3], p.wchunk_cap, wrp, nw, nc, st, ln,
                                        pr, sl);
    return placed;
}

// ---- staged (slot, vertex) appends -----------------------------------------------------

template <bool MP>
__device__ __forceinline__ void ms_flush(MsWarp<MP> &ws, unsigned n, int2 *q, unsigned *qlen, long long qcap,
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

template <bool MP>
__device__ __forceinline__ void ms_stage4(MsWarp<MP> &ws, unsigned flags, const int (&u)[4], const int (&sl)[4],
                                          int2 *q, unsigned *qlen, long long qcap, unsigned *err) {
    const unsigned lt = lanemask_lt();
    unsigned total = 0, pre[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        unsigned b = __ballot_sync(FULL, (flags >> j) & 1u);
        pre[j] = total + __popc(b & lt);
        total += __popc(b);
    }
    if (total == 0u) return;
    unsigned n = ws.nbuf;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if ((flags >> j) & 1u) ws.obuf[n + pre[j]] = make_int2(sl[j], u[j]);
    n += total;
    __syncwarp();
    if (n > unsigned(OBUF - WINDOW)) {
        ms_flush(ws, n, q, qlen, qcap, err);
        n = 0;
    }
    if (lane_id() == 0) ws.nbuf = n;
    __syncwarp();
}

// ---- direction-optimizing counts ------------------------------------------------------------

// Adds discovered vertices (bit j of disc: vertex of slot sl[j] with ln[j]
// edges) to their slots' counters of level q: lanes holding the same slot are
// grouped by __match_any_sync and their group leader adds the group's count
// and degree sum (degrees of distinct vertices of one graph: the sum stays
// below the graph's edge count, which fits in 32 bits).
__device__ __forceinline__ void count_slot_discoveries(const MsParams &p, int q, unsigned disc, const int (&ln)[4],
                                                       const int (&sl)[4]) {
    const unsigned lane = lane_id();
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const bool d = (disc >> j) & 1u;
        const unsigned peers = __match_any_sync(FULL, d ? (unsigned)sl[j] : (0x80000000u | lane));
        if (d) {
            const unsigned sum = __reduce_add_sync(peers, (unsigned)ln[j]);
            if (lane == unsigned(__ffs(peers) - 1)) {
                const size_t at = size_t(q & 3) * size_t(p.nslots) + size_t(sl[j]);
                atomicAdd(p.nf + at, unsigned(__popc(peers)));
                atomicAdd(p.mf + at, (unsigned long long)sum);
            }
        }
    }
}

// ---- the multi-search sink ---------------------------------------------------------------

// Expand-contract discovery for elements of possibly different slots: bit j
// of valid marks vertex u[j] of slot sl[j], reached from pr[j].
template <int THREADS, bool MP>
struct MsSink {
    const MsParams &p;
    MsSmem<THREADS, MP> &sm;
    int level;  // labels are level + 1 - start_level

    __device__ __forceinline__ void process(unsigned valid, const int (&u)[4], const int (&pr)[4],
                                            const int (&sl)[4]) const {
        MsSlot d[4];
        unsigned w[4], bit[4], m[4];
        const bool history = p.cull_flags & CULL_HISTORY;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            bool ok = (valid >> j) & 1u;
            d[j] = ok ? load_slot(p, sl[j]) : MsSlot{};
            if (ok && (unsigned)u[j] >= (unsigned)d[j].nodes) {
                atomicOr(&p.ctr->error, ERR_BAD_VERTEX);
                valid &= ~(1u << j);
                ok = false;
            }
            w[j] = ok ? unsigned(d[j].mask_off) + ((unsigned)u[j] >> 5) : 0u;
            bit[j] = 1u << ((unsigned)u[j] & 31u);
            if (ok && history) {
                const unsigned long long e = sm.vcache[vcache_slot(w[j])];
                if (unsigned(e >> 32) == w[j] && (unsigned(e) & bit[j])) valid &= ~(1u << j);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) m[j] = ((valid >> j) & 1u) ? ld_cg(p.mask + w[j]) : 0u;
        unsigned need = 0;
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (((valid >> j) & 1u) && !(m[j] & bit[j])) need |= 1u << j;
        unsigned old[4];
#pragma unroll
        for (int j = 0; j < 4; j++) old[j] = ((need >> j) & 1u) ? atomicOr(p.mask + w[j], bit[j]) : m[j];
        unsigned disc = 0;
        int st[4], ln[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            st[j] = 0;
            ln[j] = 0;
            if ((valid >> j) & 1u) {
                if (history) sm.vcache[vcache_slot(w[j])] = ((unsigned long long)w[j] << 32) | (old[j] | bit[j]);
                if (!(old[j] & bit[j])) {
                    disc |= 1u << j;
                    p.labels[d[j].label_off + u[j]] = MP ? pr[j] : level + 1 - d[j].start_level;
                    const int *row = p.graphs[d[j].graph].row;
                    st[j] = __ldg(row + u[j]);
                    ln[j] = __ldg(row + u[j] + 1) - st[j];
                    mark_alive(p, level + 1, sl[j]);
                }
            }
        }
        if (p.do_alpha) count_slot_discoveries(p, level + 1, disc, ln, sl);
        const unsigned enq = disc & ~ms_place4<THREADS>(p, level + 1, disc, st, ln, u, sl);
        const int nq = (level + 1) & 1;
        ms_stage4(sm.w[threadIdx.x >> 5], enq, u, sl, p.queue[nq], &p.ctr->qlen[(level + 1) & 3], p.qcap,
                  &p.ctr->error);
    }
};

// The gather_list sink interface (pred per element, out ignored) for a list
// whose elements all belong to one slot.
template <int THREADS, bool MP>
struct MsSlotSink {
    const MsSink<THREADS, MP> &s;
    int slot;
    __device__ __forceinline__ void operator()(unsigned valid, const int (&u)[4], const int (&pr)[4],
                                               unsigned) const {
        const int sl[4] = {slot, slot, slot, slot};
        s.process(valid, u, pr, sl);
    }
};

// ---- level body ---------------------------------------------------------------------------

template <int THREADS, bool MP>
__device__ void ms_level(const MsParams &p, int L, unsigned nq_in, unsigned nch, unsigned nwch,
                         MsSmem<THREADS, MP> &sm, uint64_t pol) {
    const MsSink<THREADS, MP> sink{p, sm, L};
    // CTA chunks, statically interleaved over CTAs.
    {
        unsigned n = min(nch, (unsigned)p.chunk_cap);
        const int4 *t = p.chunks[L & 1];
        for (unsigned k = blockIdx.x; k < n; k += gridDim.x) {
            const int4 c = __ldcg(t + k);
            if (c.y <= 0 || (p.do_alpha && p.bu[c.w])) continue;  // a bottom-up slot sweeps its mask instead
            const MsGraph g = p.graphs[load_slot(p, c.w).graph];
            MsSlotSink<THREADS, MP> ss{sink, c.w};
            gather_list<THREADS>(g.col, g.vec_end, c.x, c.y, c.z, 0u, threadIdx.x, ss, pol);
        }
    }
    // Warp chunks, statically interleaved over warps.
    {
        unsigned n = min(nwch, (unsigned)p.wchunk_cap);
        const int4 *t = p.wchunks[L & 1];
        const unsigned W = grid_warps();
        for (unsigned k = global_warp(); k < n; k += W) {
            const int4 c = __ldcg(t + k);
            if (c.y <= 0 || (p.do_alpha && p.bu[c.w])) continue;
            const MsGraph g = p.graphs[load_slot(p, c.w).graph];
            MsSlotSink<THREADS, MP> ss{sink, c.w};
            gather_list<32>(g.col, g.vec_end, c.x, c.y, c.z, 0u, lane_id(), ss, pol);
        }
    }
    // Frontier tiles of 32 (slot, vertex) entries, handed out dynamically.
    MsWarp<MP> &ws = sm.w[threadIdx.x >> 5];
    const int2 *q_in = p.queue[L & 1];
    const unsigned ntiles = (nq_in + 31) / 32;
    for (;;) {
        unsigned t = 0;
        if (lane_id() == 0) t = atomicAdd(&p.ctr->steal[L & 3], 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= ntiles) break;
        const unsigned idx = t * 32 + lane_id();
        int slot = 0, v = -1, start = 0, len = 0;
        const int *col = nullptr;
        int vec_end = 0;
        if (idx < nq_in && !(p.do_alpha && p.bu[__ldcg(&q_in[idx].x)])) {
            const int2 e = __ldcg(q_in + idx);
            slot = e.x;
            v = e.y;
            const MsGraph g = p.graphs[load_slot(p, slot).graph];
            start = __ldg(g.row + v);
            len = __ldg(g.row + v + 1) - start;
            col = g.col;
            vec_end = g.vec_end;
        }
        // Lists that could not be placed in chunks: streamed by the warp.
        unsigned wm;
        while ((wm = __ballot_sync(FULL, len >= p.warp_th)) != 0u) {
            const int ld = __ffs(wm) - 1;
            const int s0 = __shfl_sync(FULL, start, ld), l0 = __shfl_sync(FULL, len, ld);
            const int v0 = __shfl_sync(FULL, v, ld), sl0 = __shfl_sync(FULL, slot, ld);
            const int ve = __shfl_sync(FULL, vec_end, ld);
            const int *c0 = (const int *)__shfl_sync(FULL, (unsigned long long)col, ld);
            if ((int)lane_id() == ld) len = 0;
            MsSlotSink<THREADS, MP> ss{sink, sl0};
            gather_list<32>(c0, ve, s0, l0, v0, 0u, lane_id(), ss, pol);
        }
        // Short lists: warp prefix sum into the window of column addresses.
        const int incl = warp_inclusive_scan(len);
        const int total = __shfl_sync(FULL, incl, 31);
        const int excl = incl - len;
        for (int base = 0; base < total; base += WINDOW) {
            const int lo = max(excl, base), hi = min(excl + len, base + WINDOW);
            for (int j = lo; j < hi; j++) {
                ws.gaddr[j - base] = col + start + (j - excl);
                ws.gslot[j - base] = slot;
                if (MP) ws.gpred[j - base] = v;
            }
            __syncwarp();
            const int cnt = min(WINDOW, total - base);
            const int k = lane_id() * 4;
            unsigned valid = 0;
            int u[4], pv[4], sl[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                u[j] = -1;
                pv[j] = 0;
                sl[j] = 0;
                if (k + j < cnt) {
                    valid |= 1u << j;
                    u[j] = __ldg(ws.gaddr[k + j]);
                    sl[j] = ws.gslot[k + j];
                    pv[j] = MP ? ws.gpred[k + j] : 0;
                }
            }
            sink.process(valid, u, pv, sl);
            __syncwarp();
        }
    }
    const unsigned n = ws.nbuf;
    if (n) ms_flush(ws, n, p.queue[(L + 1) & 1], &p.ctr->qlen[(L + 1) & 3], p.qcap, &p.ctr->error);
    if (lane_id() == 0) ws.nbuf = 0;
    __syncwarp();
}

// ---- bottom-up levels ------------------------------------------------------------------

// Bottom-up step of slot s (direction-optimizing BFS, Beamer, Asanovic and
// Patterson, SC 2012; the single-search bu_step of bfs_kernels.cu with slot
// offsets): mask words w0 .. w0+3 of the slot; lane j owns vertex 32w + j of
// each word, probes its heaviest neighbour and, when that is not a parent,
// scans its list 2 entries per round, software-pipelined, for a neighbour at
// the slot's depth L - start_level.  Unlike the single search it scans per
// lane, not by warp windows: the batches' graphs are small and their lists
// short, and windows measured slower there.  Label probes are ordinary
// (L1-cached) loads, ordered after the labels they look for by the grid
// barriers before the level.  A word has one writer in the level.
template <int THREADS, bool MP>
__device__ __forceinline__ void ms_bu_step(const MsParams &p, int L, int s, unsigned w0, MsWarp<MP> &ws) {
    const MsSlot d = load_slot(p, s);
    const MsGraph g = p.graphs[d.graph];
    const unsigned nwords = (unsigned(d.nodes) + 31u) >> 5;
    unsigned *mask = p.mask + d.mask_off;
    int *labels = p.labels + d.label_off;
    const int depth = L - d.start_level;
    const int lane = lane_id();
    unsigned mw[4];
#pragma unroll
    for (int j = 0; j < 4; j++) mw[j] = w0 + j < nwords ? ld_cg(mask + w0 + j) : FULL;
    if (mw[0] == FULL && mw[1] == FULL && mw[2] == FULL && mw[3] == FULL) return;  // warp-uniform
    int v[4], st[4], ln[4];
    unsigned open = 0, scan = 0, found = 0;
    // Row offsets and the heaviest neighbour of every open vertex, loaded
    // together (a closed lane reads entry 0); the heaviest neighbour is probed
    // first, and only the vertices it does not settle read their list.
    int r0[4], r1[4];
    unsigned long long hk[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        v[j] = int((w0 + j) * 32u) + lane;
        if (v[j] < d.nodes && !((mw[j] >> lane) & 1u)) open |= 1u << j;
        const int vv = ((open >> j) & 1u) ? v[j] : 0;
        r0[j] = __ldg(g.row + vv);
        r1[j] = __ldg(g.row + vv + 1);
        hk[j] = g.heavy ? __ldg(g.heavy + vv) : 0ull;
    }
    unsigned hact = 0;
    int hp[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        st[j] = r0[j];
        ln[j] = ((open >> j) & 1u) ? r1[j] - r0[j] : 0;
        const unsigned x = unsigned(hk[j]);
        const bool a = ((open >> j) & 1u) && ln[j] > 0 && hk[j] != 0ull && x < (unsigned)d.nodes;
        if (a) hact |= 1u << j;
        hp[j] = __ldca(labels + (a ? x : 0u));
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (((hact >> j) & 1u) && hp[j] == depth) found |= 1u << j;
        // a list of one entry was settled by the probe of that entry
        if (((open >> j) & 1u) && !((found >> j) & 1u) && ln[j] > int((hact >> j) & 1u)) scan |= 1u << j;
    }
    int u[4][2];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int e = 0; e < 2; e++) u[j][e] = ((scan >> j) & 1u) && e < ln[j] ? __ldg(g.col + st[j] + e) : -1;
    for (int k = 0; __any_sync(FULL, scan != 0u); k += 2) {
        int un[4][2];
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 2; e++)
                un[j][e] = ((scan >> j) & 1u) && k + 2 + e < ln[j] ? __ldg(g.col + st[j] + k + 2 + e) : -1;
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int e = 0; e < 2; e++) {
                if (((scan >> j) & 1u) && k + e < ln[j]) {
                    const unsigned x = (unsigned)u[j][e];
                    if (x < (unsigned)d.nodes) {
                        if (__ldca(labels + x) == depth) found |= 1u << j;
                    } else {
                        atomicOr(&p.ctr->error, ERR_BAD_VERTEX);
                    }
                }
            }
            if (((found >> j) & 1u) || k + 2 >= ln[j]) scan &= ~(1u << j);
        }
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 2; e++) u[j][e] = un[j][e];
    }
    unsigned nfound = 0, dfound = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const bool f = (found >> j) & 1u;
        const unsigned fb = __ballot_sync(FULL, f);
        const unsigned zb = __ballot_sync(FULL, ((open >> j) & 1u) && ln[j] == 0);
        if (lane == 0 && (fb | zb)) __stcg(mask + w0 + j, mw[j] | fb | zb);
        if (f) {
            labels[v[j]] = depth + 1;
            nfound++;
            dfound += unsigned(ln[j]);
        }
    }
    nfound = __reduce_add_sync(FULL, nfound);
    dfound = __reduce_add_sync(FULL, dfound);
    if (nfound == 0u) return;  // warp-uniform
    if (lane == 0) {
        const size_t at = size_t((L + 1) & 3) * size_t(p.nslots) + size_t(s);
        atomicAdd(p.nf + at, nfound);
        atomicAdd(p.mf + at, (unsigned long long)dfound);
        mark_alive(p, L + 1, s);
    }
    const int sl[4] = {s, s, s, s};
    const unsigned placed = ms_place4<THREADS>(p, L + 1, found, st, ln, v, sl);
    ms_stage4(ws, found & ~placed, v, sl, p.queue[(L + 1) & 1], &p.ctr->qlen[(L + 1) & 3], p.qcap, &p.ctr->error);
}

// The bottom-up steps of every bottom-up slot, numbered in slot order by
// bu_prefix, go out in runs of R consecutive steps (R grows with the total so
// that a warp takes about 8 runs: many large slots would otherwise make the
// run counter a hot spot); the first run per warp is static, the rest are
// handed out by the counter, asked for when the previous run starts.  A run's
// slot is found by binary search and followed across slot boundaries.
template <int THREADS, bool MP>
__device__ void ms_bu_level(const MsParams &p, int L, MsWarp<MP> &ws) {
    const unsigned total = __ldcg(p.bu_prefix + p.nslots);
    const unsigned W = grid_warps();
    const unsigned R = max(1u, total / (8u * W));
    const unsigned runs = (total + R - 1) / R;
    for (unsigned r = global_warp(); r < runs;) {
        unsigned nxt = 0;
        if (runs > W && lane_id() == 0) nxt = atomicAdd(&p.ctr->bu_steal[L & 3], 1u);
        const unsigned g0 = r * R, g1 = min(total, g0 + R);
        int lo = 0, hi = p.nslots;  // last s with bu_prefix[s] <= g0
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldcg(p.bu_prefix + mid) <= g0) lo = mid;
            else hi = mid;
        }
        unsigned s_begin = __ldcg(p.bu_prefix + lo), s_end = __ldcg(p.bu_prefix + lo + 1);
        for (unsigned g = g0; g < g1; g++) {
            while (g >= s_end) {  // next slot with steps
                lo++;
                s_begin = s_end;
                s_end = __ldcg(p.bu_prefix + lo + 1);
            }
            ms_bu_step<THREADS, MP>(p, L, lo, (g - s_begin) * 4u, ws);
        }
        r = runs > W ? W + __shfl_sync(FULL, nxt, 0) : runs;
    }
}

// Direction of level L for every slot (block 0, before the level's work):
// the rule of the single-search DirectionChoice applied to the slot's counts,
// then bu_prefix as an exclusive scan of the bottom-up slots' step counts.
// Also clears the counts level L+1 will fill into ring entry (L+2)&3.
template <int THREADS, bool MP>
__device__ void ms_directions(const MsParams &p, int L, MsSmem<THREADS, MP> &sm) {
    __syncthreads();
    const unsigned char *in = p.alive + size_t(L & 3) * size_t(p.nslots);
    const MsDir *prev = p.dir + size_t((L + 1) & 1) * size_t(p.nslots);  // state after level L-1
    MsDir *next = p.dir + size_t(L & 1) * size_t(p.nslots);
    unsigned carry = 0;
    // Rounds of THREADS consecutive slots (coalesced loads), each closed by a
    // block-wide exclusive scan of the bottom-up steps.
    for (int r0 = 0; r0 < p.nslots; r0 += THREADS) {
        const int s = r0 + int(threadIdx.x);
        unsigned steps = 0;
        if (s < p.nslots) {
            const size_t at = size_t(L & 3) * size_t(p.nslots) + size_t(s);
            const size_t clr = size_t((L + 2) & 3) * size_t(p.nslots) + size_t(s);
            const bool live = !MP && in[s] && p.state[s].active;
            bool bottom_up = false;
            if (live) {
                MsDir dr = prev[s];
                const unsigned nf = p.nf[at];
                const unsigned long long mf = p.mf[at];
                dr.explored += mf;
                dr.visited += nf;
                if (dr.symmetric) {
                    const unsigned long long total = (unsigned long long)dr.edges;
                    const unsigned long long unexplored = total > dr.explored ? total - dr.explored : 0ull;
                    if (!dr.bottom_up) bottom_up = mf * p.do_alpha > unexplored;
                    else bottom_up = !((unsigned long long)nf * p.do_beta < (unsigned long long)dr.nodes && nf < dr.prev_nf);
                }
                dr.prev_nf = nf;
                dr.bottom_up = bottom_up ? 1 : 0;
                next[s] = dr;
                if (bottom_up) steps = ((unsigned(dr.nodes) + 31u) / 32u + 3u) / 4u;
            }
            p.nf[clr] = 0u;
            p.mf[clr] = 0ull;
            p.bu[s] = bottom_up ? 1 : 0;
        }
        const unsigned incl = (unsigned)warp_inclusive_scan(int(steps));
        if (lane_id() == 31) sm.warp_tot[threadIdx.x >> 5] = incl;
        __syncthreads();
        unsigned base = carry, round_total = 0;
        for (int w = 0; w < THREADS / 32; w++) {
            if (w < int(threadIdx.x >> 5)) base += sm.warp_tot[w];
            round_total += sm.warp_tot[w];
        }
        if (s < p.nslots) p.bu_prefix[s] = base + incl - steps;
        carry += round_total;
        __syncthreads();  // warp_tot is rewritten by the next round
    }
    if (threadIdx.x == 0) {
        p.bu_prefix[p.nslots] = carry;
        p.ctr->bu_steal[L & 3] = 0u;
    }
    __syncthreads();
}

// One CTA retires the slots without input for level L and clears the alive
// entries level L+1 will fill.  final_sweep: the batch has no work left, so
// every active slot ends here.
// Retired searches are counted in Counters::retired[L&3] (zeroed at level L-1).
__device__ void ms_bookkeeping(const MsParams &p, int L, bool final_sweep) {
    const unsigned char *in = p.alive + size_t(L & 3) * size_t(p.nslots);
    unsigned char *clear = p.alive + size_t((L + 2) & 3) * size_t(p.nslots);
    const unsigned long long now = globaltimer_ns();
    unsigned retired = 0;
    if (threadIdx.x == 0) p.ctr->retired[(L + 1) & 3] = 0u;
    for (int s = threadIdx.x; s < p.nslots; s += blockDim.x) {
        MsSlotState &st = p.state[s];
        if (st.active && (final_sweep || !in[s])) {
            st.active = 0;
            st.done_levels = L - load_slot(p, s).start_level;
            st.done_ns = now;
            retired++;
        }
        clear[s] = 0;
    }
    if (retired) atomicAdd(&p.ctr->retired[L & 3], retired);
}

__device__ __forceinline__ void ms_ring_prepare(Counters *c, int q) {
    c->qlen[(q + 2) & 3] = 0u;
    c->big[(q + 2) & 3] = 0u;
    c->wch[(q + 2) & 3] = 0u;
    c->steal[(q + 1) & 3] = 0u;
}

template <int THREADS, bool MP>
__global__ void __launch_bounds__(THREADS, MS_MIN_BLOCKS(THREADS)) ms_fused_kernel(MsParams p) {
    MsSmem<THREADS, MP> &sm = ms_smem<THREADS, MP>();
    if (lane_id() == 0) sm.w[threadIdx.x >> 5].nbuf = 0;
    if (p.cull_flags & CULL_HISTORY)
        for (int i = threadIdx.x; i < VCACHE; i += THREADS) sm.vcache[i] = ~0ull << 32;
    __syncthreads();
    const uint64_t pol = policy_evict_first();
    Counters *c = p.ctr;
    int L = c->cur_it;
    const int L_end = p.max_levels > 0 ? L + p.max_levels : 0x7fffffff;
    const int L_first = L;
    // A level's counts are loaded by one thread per CTA and shared (a load per
    // thread would send every warp of the grid to the same L2 lines): for the
    // first level here, for the others by the grid barrier before them.
    // Retired: searches retired at the previous level's start (final before
    // the barrier).
    if (threadIdx.x == 0) sm.lc = load_counts(c, L, false);
    __syncthreads();
    for (;;) {
        const unsigned nq = sm.lc.L, nch = sm.lc.nch, nw = sm.lc.nw;
        const bool retired_before = sm.lc.retired != 0u;
        const bool empty = nq + nch + nw == 0u;
        if (blockIdx.x == 0) ms_bookkeeping(p, L, empty);
        if (empty || L >= L_end || (p.stop_on_retire && retired_before)) break;
        // Direction-optimizing: every CTA needs the level's per-slot directions
        // before it takes any work.  The last CTA to reach the previous level's
        // barrier decides them; a launch's first level decides them behind a
        // barrier of its own (deciding a level again gives the same result:
        // the state read is that of the level before, in the other half of
        // dir).
        if (p.do_alpha && L == L_first) {
            if (blockIdx.x == 0) ms_directions<THREADS, MP>(p, L, sm);
            if (!grid_barrier(c, p.wait_ns, &sm.flag)) break;
        }
        if (leader()) {
            ms_ring_prepare(c, L);
            if (p.levels && L < p.level_cap) {
                LevelRecord r;
                r.t_start = globaltimer_ns();
                r.frontier = nq;
                r.chunks = nch;
                r.wchunks = nw;
                r.bottom_up = 0;
                p.levels[L] = r;
            }
        }
        ms_level<THREADS, MP>(p, L, nq, nch, nw, sm, pol);
        if constexpr (!MP) {  // bottom-up levels test depth labels
            if (p.do_alpha) {
                MsWarp<MP> &ws = sm.w[threadIdx.x >> 5];
                ms_bu_level<THREADS, MP>(p, L, ws);
                const unsigned n = ws.nbuf;
                if (n) ms_flush(ws, n, p.queue[(L + 1) & 1], &c->qlen[(L + 1) & 3], p.qcap, &c->error);
                if (lane_id() == 0) ws.nbuf = 0;
                __syncwarp();
            }
        }
        const NextCounts next = next_counts(&sm.lc, L + 1, false, true);
        if (p.do_alpha) {
            if (!grid_barrier_serial(c, p.wait_ns, &sm.flag, &sm.last,
                                     [&] { ms_directions<THREADS, MP>(p, L + 1, sm); }, &next))
                break;
        } else if (!grid_barrier(c, p.wait_ns, &sm.flag, gridDim.x, &next)) {
            break;
        }
        L++;
    }
    if (leader()) {
        c->cur_it = L;
        atomicOr(&c->sticky, ld_relaxed_gpu(&c->error));
    }
}

// Admission: one thread per new (slot, source).  Labels and mask of the slot
// are already cleared; the source is labelled, marked and its list placed as
// input of level cur_it like any discovered vertex's list.
template <int THREADS>
__global__ void ms_admit_kernel(MsParams p, const int2 *slot_src, int count, int mark_pred) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Counters *c = p.ctr;
    const int L = c->cur_it;
    const int slot = slot_src[i].x, src = slot_src[i].y;
    const MsSlot d = load_slot(p, slot);
    if ((unsigned)src >= (unsigned)d.nodes) {
        atomicOr(&c->error, ERR_BAD_VERTEX);
        return;
    }
    p.labels[d.label_off + src] = mark_pred ? -2 : 0;
    atomicOr(p.mask + unsigned(d.mask_off) + (unsigned(src) >> 5), 1u << (unsigned(src) & 31u));
    MsSlotState st;
    st.active = 1;
    st.done_levels = -1;
    st.done_ns = 0;
    p.state[slot] = st;
    p.alive[size_t(L & 3) * size_t(p.nslots) + slot] = 1;
    const MsGraph g = p.graphs[d.graph];
    const int start = g.row[src], len = g.row[src + 1] - start;
    if (p.do_alpha) {
        MsDir dr = {};
        dr.nodes = g.nodes;
        dr.edges = g.edges;
        dr.symmetric = g.symmetric;
        p.dir[slot] = dr;
        p.dir[size_t(p.nslots) + size_t(slot)] = dr;
        for (int q = 0; q < 4; q++) {
            const size_t at = size_t(q) * size_t(p.nslots) + size_t(slot);
            p.nf[at] = q == (L & 3) ? 1u : 0u;
            p.mf[at] = q == (L & 3) ? (unsigned long long)len : 0ull;
        }
    }
    constexpr int CH = chunk_edges<THREADS>();
    const bool cta = len >= p.cta_th, wrp = !cta && len >= p.warp_th;
    if (cta || wrp) {
        const int chs = cta ? CH : WARP_CHUNK;
        const int a0 = start & ~3, nch = (start + len - a0 + chs - 1) / chs;
        unsigned *count_p = cta ? &c->big[L & 3] : &c->wch[L & 3];
        const unsigned base = atomicAdd(count_p, unsigned(nch));
        const int cap = cta ? p.chunk_cap : p.wchunk_cap;
        int4 *table = (cta ? p.chunks : p.wchunks)[L & 1];
        if ((long long)base + nch <= cap) {
            for (int k = 0; k < nch; k++) {
                const int ws = a0 + k * chs;
                const int cs = max(ws, start), ce = min(ws + chs, start + len);
                table[base + k] = make_int4(cs, ce - cs, src, slot);
            }
            return;
        }
        for (long long k = base; k < cap && k < (long long)base + nch; k++) table[k] = make_int4(0, 0, 0, 0);
    }
    const unsigned pos = atomicAdd(&c->qlen[L & 3], 1u);
    if (pos < (unsigned long long)p.qcap) p.queue[L & 1][pos] = make_int2(slot, src);
    else atomicOr(&c->error, ERR_OVERFLOW);
}

// One CTA per slot: labels := -1 and visited-mask words := 0.
__global__ void ms_clear_kernel(MsParams p, const int *slots, int count) {
    if ((int)blockIdx.x >= count) return;
    const MsSlot d = load_slot(p, slots[blockIdx.x]);
    int *labels = p.labels + d.label_off;
    unsigned *mask = p.mask + d.mask_off;
    const int words = (d.nodes + 31) / 32;
    for (int i = threadIdx.x; i < d.nodes; i += blockDim.x) labels[i] = -1;
    for (int i = threadIdx.x; i < words; i += blockDim.x) mask[i] = 0u;
}

typedef void (*MsKernelFn)(MsParams);

template <bool MP>
MsKernelFn ms_fn(int threads, size_t *smem) {
    switch (threads) {
    case 128: *smem = sizeof(MsSmem<128, MP>); return ms_fused_kernel<128, MP>;
    case 512: *smem = sizeof(MsSmem<512, MP>); return ms_fused_kernel<512, MP>;
    default: *smem = sizeof(MsSmem<256, MP>); return ms_fused_kernel<256, MP>;
    }
}

MsKernelFn pick(const MsKernelConfig &kc, size_t *smem) {
    return kc.mark_pred ? ms_fn<true>(kc.threads, smem) : ms_fn<false>(kc.threads, smem);
}

}  // namespace

cudaError_t ms_graph_symmetric(const int *d_row, const int *d_col, int nodes, long long edges, int *symmetric) {
    unsigned long long *d = nullptr, h[4] = {0, 0, 0, 0};
    cudaError_t e = cudaMalloc(&d, sizeof(h));
    if (!e) e = cudaMemset(d, 0, sizeof(h));
    if (!e) e = launch_symmetry_hash(d_row, d_col, nodes, edges, d, 0);
    if (!e) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (!e) *symmetric = (h[0] == h[1] && h[2] == h[3]) ? 1 : 0;
    return e;
}

cudaError_t ms_graph_heavy(const int *d_row, const int *d_col, int nodes, long long edges, unsigned long long **keys) {
    *keys = nullptr;
    if (nodes <= 0) return cudaSuccess;
    unsigned long long *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long) * size_t(nodes));
    if (!e) e = cudaMemset(d, 0, sizeof(unsigned long long) * size_t(nodes));
    if (!e) e = launch_heavy_neighbour(d_row, d_col, nodes, edges, d, 0);
    if (!e) e = cudaStreamSynchronize(0);
    if (e) {
        cudaFree(d);
        return e;
    }
    *keys = d;
    return cudaSuccess;
}

cudaError_t ms_grid_limit(const MsKernelConfig &kc, int *grid) {
    size_t smem = 0;
    MsKernelFn fn = pick(kc, &smem);
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (!e) e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)fn, kc.threads, smem);
    if (e) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    *grid = sms * occ;
    return cudaSuccess;
}

cudaError_t ms_launch(const MsParams &p, const MsKernelConfig &kc, int grid, cudaStream_t stream) {
    size_t smem = 0;
    MsKernelFn fn = pick(kc, &smem);
    cudaError_t e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kc.threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, fn, p);
}

cudaError_t ms_clear_slots(const MsParams &p, const int *d_slots, int count, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    ms_clear_kernel<<<count, 512, 0, stream>>>(p, d_slots, count);
    return cudaGetLastError();
}

cudaError_t ms_admit(const MsParams &p, const MsKernelConfig &kc, const int2 *d_slot_src, int count,
                     cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int blocks = (count + 127) / 128;
    const int mp = kc.mark_pred ? 1 : 0;
    switch (kc.threads) {
    case 128: ms_admit_kernel<128><<<blocks, 128, 0, stream>>>(p, d_slot_src, count, mp); break;
    case 512: ms_admit_kernel<512><<<blocks, 128, 0, stream>>>(p, d_slot_src, count, mp); break;
    default: ms_admit_kernel<256><<<blocks, 128, 0, stream>>>(p, d_slot_src, count, mp); break;
    }
    return cudaGetLastError();
}

}  // namespace b40c_b200
