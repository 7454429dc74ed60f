// Device-side building blocks of the B200 BFS kernels (sm_100a).
//
// Replaces b40c/util/{global_barrier,cta_work_progress,io/*,scan/*}.cuh with
// sm_100 idioms:
//   * a grid barrier of one arrival counter and a generation word, with
//     release/acquire at GPU scope and a %globaltimer spin limit, in place of
//     GlobalBarrier::Sync (util/global_barrier.cuh:80-126), which polls one
//     flag per CTA from block 0 and spins without bound;
//   * queue/steal/big-list counters in a 4-entry ring indexed by iteration,
//     as CtaWorkProgress keeps queue counters at [iteration & 3]
//     (util/cta_work_progress.cuh:69-223);
//   * warp-shuffle scans in place of the raking smem scans
//     (util/scan/cooperative_scan.cuh:173-195);
//   * visited-bitmask culling with atomicOr, which makes the mask exact (the
//     reference's mask store is a best-effort race, contract_expand_atomic/
//     cta.cuh:213-258, backed by a label check, :264-304).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace b40c_b200 {

// ---- error bits raised on the device (Counters::error) ----------------------
enum : unsigned {
    ERR_OVERFLOW = 1u,         // frontier queue capacity exceeded
    ERR_BARRIER_TIMEOUT = 2u,  // a grid barrier wait ran past its limit
    ERR_BAD_VERTEX = 4u,       // a column index >= nodes (malformed CSR)
    ERR_LEVEL_LIMIT = 8u,      // more levels than vertices: visited state inconsistent
};

// A BFS has at most nodes levels; the level loops stop (with ERR_LEVEL_LIMIT)
// past this bound so no persistent kernel can spin without end.
__device__ __forceinline__ bool level_limit_hit(int it, int nodes) { return it > nodes + 2; }

// Per-search device counters.  ring[x][it & 3] as CtaWorkProgress does.
// Every group of counters that takes atomics lives in its own 256-byte block,
// so that their atomics are served by different L2 slices instead of queueing
// at one.
struct alignas(256) Counters {
    unsigned qlen[4];    // qlen[q&3]: length of the input frontier queue of phase q
    unsigned pad_q[60];
    unsigned steal[4];   // steal[q&3]: next warp tile to hand out in phase q
    unsigned pad_s[60];
    unsigned big[4];     // big[q&3]: CTA chunks of neighbour lists input to phase q
    unsigned pad_b[60];
    unsigned wch[4];     // wch[q&3]: warp chunks of neighbour lists input to phase q
    unsigned pad_w[60];
    // raw[q&3]: the edge frontier phase q has as the reference defines it --
    // every neighbour of the vertices the phase before expanded, whether it
    // sits in the queue, in a chunk, or was dropped by the gather-time cull.
    // Edge-frontier strategies stop, count total_queued and log by it.
    unsigned raw[4];
    unsigned pad_r[60];
    unsigned error;      // ERR_* bits
    int iteration;       // iteration counter at exit (reference d_iteration)
    int cur_it;          // current iteration for per-level (graph-driven) kernels
    unsigned done;       // 1 once the search has finished (per-level variants)
    unsigned long long total_queued;  // sum of frontier lengths (instrumented)
    unsigned retired[4];  // multi-search: searches retired at the start of level q, at [q&3]
    int resume;           // level a full-grid fused launch starts at (set by a narrow launch before it)
    // Expand-contract direction-switch state before level `resume` (set by a
    // narrow launch with the handover; see DirectionChoice).
    unsigned dir_visited, dir_prev_nf, dir_bottom_up;
    unsigned long long dir_explored;
    unsigned pad_e[48];
    // Direction-optimizing expand-contract: the vertices discovered as input of
    // phase q (mf: the sum of their degrees, nf: their number), at [q&3].
    unsigned long long mf[4];
    unsigned nf[4];
    unsigned zmarked;  // vertices without edges that bottom-up levels marked visited (whole search)
    unsigned bu_steal[4];  // multi-search: next bottom-up step of level q, at [q&3]
    unsigned pad_f[47];
    unsigned bar_count;  // grid_barrier_serial: arrivals of the current barrier
    unsigned bar_gen;    // grid_barrier_serial: generation
    unsigned long long bar_total;  // grid_barrier: arrivals since the counters were cleared
    unsigned pad_g[59];
    unsigned sticky;  // OR of error over searches since the host last read it (not reset per search)
};
// Each group of counters above fills its own 256-byte block: a new field
// takes padding of its block, never the next block's place.
static_assert(sizeof(Counters) == 2048, "Counters: 8 blocks of 256 bytes");
static_assert(offsetof(Counters, error) == 1280 && offsetof(Counters, mf) == 1536 &&
                  offsetof(Counters, bar_count) == 1792 && offsetof(Counters, sticky) == 2044,
              "Counters: block boundaries");

// ---- PTX helpers ---------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_gpu(unsigned *p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acqrel_gpu(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long atom_add_acqrel_gpu_u64(unsigned long long *p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// L2-coherent load of data written by other CTAs during this kernel (skips L1).
__device__ __forceinline__ int ld_cg(const int *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_cg(const unsigned *p) { return __ldcg(p); }

// L2 eviction-priority policies (createpolicy, sm_80+): stream the column
// indices through L2 with evict_first so the visited mask, labels and row
// offsets stay resident.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ int4 ldg_stream_v4(const int *p, uint64_t pol) {
    int4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ldg_stream(const int *p, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
                 : "=r"(v)
                 : "l"(p), "l"(pol));
    return v;
}

// ---- bulk copies into shared memory with mbarrier completion (sm_90+) ---------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return unsigned(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes initialised mbarriers visible to the bulk-copy unit.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Global -> shared bulk copy of `bytes` (a multiple of 16; both addresses
// 16-byte aligned) completing on mbarrier bar.  A plain (non-multicast) copy
// from this GPU's own memory.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Orders the generic-proxy global writes this thread has observed before the
// bulk (async-proxy) reads it issues next.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// The counts a fused kernel's phase starts from.
struct LevelCounts {
    unsigned L;             // input vertex or edge frontier queue length
    unsigned nch, nw;       // CTA and warp chunks of neighbour lists input to the phase
    unsigned nf;            // direction switch: vertices discovered for the phase
    unsigned zmarked;       // direction switch: vertices without edges marked so far
    unsigned retired;       // multi-search: searches retired at the previous phase's start
    unsigned raw;           // edge-frontier strategies: the phase's edge frontier before culling
    unsigned long long mf;  // direction switch: their edges
};

// Loads the counts phase q starts from (dir: with the direction counts;
// retired: with the multi-search retirements of phase q - 1).
__device__ __forceinline__ LevelCounts load_counts(const Counters *c, int q, bool dir, bool retired = false) {
    LevelCounts v;
    v.L = __ldcg(&c->qlen[q & 3]);
    v.nch = __ldcg(&c->big[q & 3]);
    v.nw = __ldcg(&c->wch[q & 3]);
    v.nf = dir ? __ldcg(&c->nf[q & 3]) : 0u;
    v.zmarked = dir ? __ldcg(&c->zmarked) : 0u;
    v.retired = retired ? __ldcg(&c->retired[(q - 1) & 3]) : 0u;
    v.raw = __ldcg(&c->raw[q & 3]);
    v.mf = dir ? __ldcg(&c->mf[q & 3]) : 0ull;
    return v;
}

// What a grid barrier loads for the phase after it: the counts of phase q,
// into the CTA's shared copy *out.
struct NextCounts {
    LevelCounts *out;
    int q;
    bool dir;
    bool retired;
};
__device__ __forceinline__ NextCounts next_counts(LevelCounts *out, int q, bool dir, bool retired = false) {
    return NextCounts{out, q, dir, retired};
}

// ---- grid barrier ----------------------------------------------------------------
// All CTAs of a cooperative launch call this the same number of times.  Each
// CTA's thread 0 arrives with an acq_rel add on a 64-bit count of all
// arrivals since the counters were cleared; the barrier it is in ends when the
// count reaches the next multiple of `expected`, which every waiting CTA sees
// directly (no last-arriver flip of a generation word, one L2 round trip
// less).  A waiting CTA spins with an acquire load until then, the error word
// becomes non-zero, or wait_ns of %globaltimer time pass (then
// ERR_BARRIER_TIMEOUT is raised and the CTA leaves the wait).  Returns false
// on any raised error, identically for every thread of the CTA.  With `next`,
// the waiting thread also loads the next phase's counts into the CTA's shared
// copy, in the same round trip as the error word: every thread reads them
// after the barrier, and no warp has to go to L2 for them.
__device__ __forceinline__ bool grid_barrier(Counters *c, unsigned long long wait_ns,
                                             unsigned *smem_flag, unsigned expected,
                                             const NextCounts *next = nullptr) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long arrived = atom_add_acqrel_gpu_u64(&c->bar_total, 1ull);
        const unsigned long long target = (arrived / expected + 1ull) * expected;
        if (arrived + 1ull != target) {
            const unsigned long long t0 = globaltimer_ns();
            unsigned ns = 16;
            while (ld_acquire_gpu_u64(&c->bar_total) < target) {
                if (ld_relaxed_gpu(&c->error) != 0u) break;
                if (globaltimer_ns() - t0 > wait_ns) {
                    atomicOr(&c->error, ERR_BARRIER_TIMEOUT);
                    break;
                }
                __nanosleep(ns);
                if (ns < 128) ns <<= 1;
            }
        }
        if (next) *next->out = load_counts(c, next->q, next->dir, next->retired);
        *smem_flag = ld_relaxed_gpu(&c->error);
    }
    __syncthreads();
    return *smem_flag == 0u;
}
__device__ __forceinline__ bool grid_barrier(Counters *c, unsigned long long wait_ns,
                                             unsigned *smem_flag) {
    return grid_barrier(c, wait_ns, smem_flag, gridDim.x);
}
__device__ __forceinline__ bool grid_barrier(Counters *c, unsigned long long wait_ns, unsigned *smem_flag,
                                             NextCounts next) {
    return grid_barrier(c, wait_ns, smem_flag, gridDim.x, &next);
}

// ---- cluster barrier -------------------------------------------------------------
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The same barrier with a serial section: the CTA whose arrival completes the
// count runs serial() with all its threads (it may use __syncthreads) before
// it publishes the new generation, so serial() sees everything every CTA did
// before the barrier and every CTA sees its results after it.
// With `next`, thread 0 of every CTA loads the next phase's counts after the
// barrier, with the error word, as grid_barrier does.
template <class F>
__device__ __forceinline__ bool grid_barrier_serial(Counters *c, unsigned long long wait_ns, unsigned *smem_flag,
                                                    unsigned *smem_last, const F &serial,
                                                    const NextCounts *next = nullptr) {
    __syncthreads();
    unsigned gen = 0;
    if (threadIdx.x == 0) {
        gen = ld_acquire_gpu(&c->bar_gen);
        const unsigned arrived = atom_add_acqrel_gpu(&c->bar_count, 1u);
        *smem_last = arrived == gridDim.x - 1 ? 1u : 0u;
    }
    __syncthreads();
    if (*smem_last) {
        serial();
        __syncthreads();
        if (threadIdx.x == 0) {
            st_relaxed_gpu(&c->bar_count, 0u);
            st_release_gpu(&c->bar_gen, gen + 1u);
        }
    } else if (threadIdx.x == 0) {
        const unsigned long long t0 = globaltimer_ns();
        unsigned ns = 32;
        while (ld_acquire_gpu(&c->bar_gen) == gen) {
            if (ld_relaxed_gpu(&c->error) != 0u) break;
            if (globaltimer_ns() - t0 > wait_ns) {
                atomicOr(&c->error, ERR_BARRIER_TIMEOUT);
                break;
            }
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
        }
    }
    if (threadIdx.x == 0) {
        if (next) *next->out = load_counts(c, next->q, next->dir, next->retired);
        *smem_flag = ld_relaxed_gpu(&c->error);
    }
    __syncthreads();
    return *smem_flag == 0u;
}

// ---- scans -------------------------------------------------------------------------
__device__ __forceinline__ int warp_sum(int x) { return __reduce_add_sync(0xffffffffu, x); }
__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
    return x;
}
__device__ __forceinline__ int warp_inclusive_scan(int x) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, d);
        if ((int)lane_id() >= d) x += y;
    }
    return x;
}

// Block-wide exclusive scan of two components at once (the reference's SoA
// scan of (coarse, fine) ranks, contract_expand_atomic/cta.cuh:624-633).
// warp_tot must hold THREADS/32 int2 in shared memory.  Ends with a barrier
// so warp_tot may be reused right after.
template <int THREADS>
__device__ __forceinline__ int2 block_exclusive_scan2(int2 v, int2 &total, int2 *warp_tot) {
    constexpr int WARPS = THREADS / 32;
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int ix = warp_inclusive_scan(v.x);
    int iy = warp_inclusive_scan(v.y);
    if (lane == 31) warp_tot[warp] = make_int2(ix, iy);
    __syncthreads();
    if (warp == 0) {
        int2 t = lane < WARPS ? warp_tot[lane] : make_int2(0, 0);
        int sx = warp_inclusive_scan(t.x);
        int sy = warp_inclusive_scan(t.y);
        if (lane < WARPS) warp_tot[lane] = make_int2(sx - t.x, sy - t.y);  // exclusive warp bases
        if (lane == WARPS - 1) warp_tot[WARPS] = make_int2(sx, sy);       // block total
    }
    __syncthreads();
    int2 base = warp_tot[warp];
    total = warp_tot[WARPS];
    __syncthreads();
    return make_int2(base.x + ix - v.x, base.y + iy - v.y);
}

template <int THREADS>
__device__ __forceinline__ int block_exclusive_scan(int v, int &total, int2 *warp_tot) {
    int2 t2;
    int2 r = block_exclusive_scan2<THREADS>(make_int2(v, 0), t2, warp_tot);
    total = t2.x;
    return r.x;
}

// ---- visited mask ------------------------------------------------------------------
// Exact test-and-set of vertex u's bit: a cheap L2 read first, and an atomicOr
// only when the bit looked clear.  Returns true for exactly one caller per
// vertex over the whole search.
__device__ __forceinline__ bool mark_visited(unsigned *mask, int u) {
    unsigned w = unsigned(u) >> 5, bit = 1u << (unsigned(u) & 31u);
    if (ld_cg(mask + w) & bit) return false;
    return (atomicOr(mask + w, bit) & bit) == 0u;
}

// ---- neighbour-list streaming -----------------------------------------------------

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
// list [s, s+l) with 16-byte loads starting from the 4-aligned index s & ~3;
// each pass covers GROUP*4 elements; the next pass's load is issued before the
// current elements are processed.  Elements outside [s, s+l) are masked off.
// No group-wide barrier: every warp of the group proceeds on its own.
template <int GROUP, class Sink>
__device__ __forceinline__ void gather_list(const int *col, int vec_end, int s, int l, int pred, unsigned out,
                                            int rank, const Sink &sink, uint64_t pol) {
    const int end = s + l;
    int e = (s & ~3) + rank * 4;
    int4 cur = load_col4(col, vec_end, e, end, pol);
    const int pv[4] = {pred, pred, pred, pred};
    for (int base = s & ~3; base < end; base += GROUP * 4) {
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

// ---- history cache -------------------------------------------------------------------
constexpr int VCACHE = 2048;  // visited-mask words held per CTA

// Slot of mask word w in the CTA's history cache (multiplicative hash, so the
// low-popcount word indices of skewed graphs spread over the slots).
__device__ __forceinline__ unsigned vcache_slot(unsigned w) { return (w * 2654435761u) >> (32 - 11); }
static_assert(VCACHE == 2048, "vcache_slot takes 11 bits");

}  // namespace b40c_b200
