// gfc_batch.cu -- many lattices at once, with per-timeslice retirement.
//
// The Coulomb gauge condition decouples timeslices: during the sweeps a timeslice
// shares no link with another.  The batch therefore schedules timeslices, not
// lattices.  Every timeslice of every resident lattice ("slot") carries a state:
//
//   FP32   bulk sweeps on two-row FP32 links and G
//   PEND   its FP32 e2 fell below the switch threshold: rebuild in FP64 next round
//   FP64   refinement on two-row FP64 links and G
//   DONE   its own e2 fell below the tolerance: retired, no more work
//
// A round is: compaction (work lists of (timeslice, 128-site chunk) items for the
// FP32 and FP64 states and of pending timeslices), the FP64 rebuild of the pending
// timeslices (G from its FP32 copy, projected; links as G U0 G^dagger from the FP64
// originals), then K half-sweeps, each one persistent FP32 kernel and one
// persistent FP64 kernel over their work lists, plus periodic reunitarisation.
// All parameters live in device memory, so one round is captured once as a CUDA
// graph and replayed; the host only reads the state table between rounds.
//
// The sweep kernels write one pair of fused-e2 partials per chunk; after each
// half-sweep k_bslice sums each timeslice's partials in a fixed order, adds the
// other parity's contribution from the previous half-sweep (ring buffer) and
// decides the switch or the retirement of that timeslice alone.
//
// Slots can be added, activated, finalised and removed between rounds, which is
// what the serving loop does (continuous batching).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gfc.h"
#include "gfc_ctx.h"
#include "gfc_fast_device.cuh"
#include "gfc_internal.h"

namespace gfc {

enum : int { SS_EMPTY = 0, SS_FP32 = 1, SS_PEND = 2, SS_FP64 = 3, SS_DONE = 4, SS_VERIFY = 5, SS_LEX = 6 };
// SS_LEX: a timeslice of an odd-ns lattice, FP64 on two stored rows in the
// lexicographic layout.  Same-parity sites meet across the periodic boundary there,
// so a half-sweep runs as four launches over the boundary levels (the number of
// coordinates equal to ns - 1), which keeps the order of the sequential z, y, x
// sweep between every pair of sites that share a link; e2 is measured by a separate
// pass over the state the half-sweep leaves (a site's post-update w is not final
// when a later level updates a neighbour), so no verify pass is needed.
// SS_VERIFY: the FP64 e2 measured after half-sweep c - 1 fell below the tolerance, but
// the timeslice has had half-sweep c too.  Its next pass measures e2 of the state it
// is in without updating it: below the tolerance -> DONE with that state, else back
// to FP64 (measured after every half-sweep).  So a retired timeslice's e2 is below
// the tolerance for the links it keeps, not for an earlier state.
// e2 of a timeslice after half-sweep c needs the fused sums of its half-sweeps c and
// c + 1.  While its target (switch threshold or tolerance) is far, a timeslice is
// measured on own half-sweep counts 30, 31 (mod 32) only; once the last measurement
// or the rate between the last two puts the target near, after every half-sweep.
enum : int { MF_NOW = 1, MF_PREV = 2, MF_DENSE = 4 };
constexpr int MEASURE_PERIOD = 32;
__host__ __device__ constexpr int measure_at(int c) { return c % MEASURE_PERIOD >= MEASURE_PERIOD - 2; }
constexpr int BCHUNK = 128;   // sites per work item = threads per CTA of the sweep kernels
constexpr int BPIECES = BCHUNK / 32;   // 32-site pieces of an item; e2 partials are kept per piece

struct BSlot {          // device-visible descriptor of one resident lattice
    Lat l;
    double2 *u, *ut, *g;   // FP64 full: canonical links and G
    double2 *u64r, *g64r;  // FP64 two-row working copies
    float4 *u32, *g32;     // FP32 two-row working copies
    double *part;          // [nt][nbx][BPIECES][2] partials of the fused e2, one pair per
                           // 32-site piece, each summed over its warp by the same shuffle
                           // tree whichever kernel and hand-out swept it
    int nbx;               // chunks per timeslice and parity = ceil(vs/2 / BCHUNK)
    int nfull;             // chunks per timeslice over both parities = ceil(vs / BCHUNK)
};

struct BState {
    BSlot *slots;
    int max_nt, nslices;
    int *state;           // [nslices], gid = slot * max_nt + t
    int *sweeps;          // [nslices] half-sweeps applied to the timeslice
    int *listed;          // [nslices] 1 if this round's sweep work lists hold the timeslice
    const int *held;      // [max_slots] 1: the slot is resident but kept out of the rounds
    int *mflag;           // [nslices] e2 measurement: MF_NOW, MF_PREV, MF_DENSE
    int *mk;              // [nslices] own half-sweep count of the last e2 measurement (-1: none)
    double *me2;          // [nslices] that e2
    double *ring;         // [2][nslices][2]: (pre, post) e2 sums of the last two half-sweeps
    int2 *items32, *items64, *pend, *itemslex;
    int cap_items, cap_pend;
    int lex;              // 1: odd-ns slots may be active (their launches are in the round)
    int *counts;          // [0] n32 [1] n64 [2] npend [3] active timeslices [4] half-sweep k [5] overflow
                          // [6] [7] item cursors [8] [9] FP32 / FP64 reunitarisation due
                          // [10] nlex [11..14] cursors of the odd-ns levels [15] of the odd-ns e2 pass
                          // [16] an FP32 rebuild due
    unsigned *status;
    double omega, switch_e2, tol;
    unsigned hits, reunit32, reunit64;
    unsigned refresh32;   // options.fp32_refresh: rebuild the FP32 fields every n own half-sweeps
};

// ------------------------------------------------------------------ compaction --
// One block.  Builds the three work lists from the state table.
__global__ void __launch_bounds__(1024) k_compact(BState b) {
    __shared__ int sc[4][1024];
    __shared__ int sact[1024];
    const int tid = threadIdx.x;
    const int per = (b.nslices + 1023) / 1024;
    const int g0 = tid * per, g1 = min(g0 + per, b.nslices);
    int c[4] = {0, 0, 0, 0}, act = 0;
    for (int gid = g0; gid < g1; gid++) {
        int st = b.state[gid];
        const bool held = b.held[gid / b.max_nt];
        b.listed[gid] = !held && (st == SS_FP32 || st == SS_FP64 || st == SS_VERIFY || st == SS_LEX);
        if (st == SS_EMPTY || st == SS_DONE) continue;
        const BSlot &sl = b.slots[gid / b.max_nt];
        act++;
        if (held) continue;   // frozen: no items, no switch this round
        if (st == SS_FP32) c[0] += sl.nbx;
        else if (st == SS_FP64 || st == SS_VERIFY) c[1] += sl.nbx;
        else if (st == SS_PEND) c[2] += sl.nfull;
        else if (st == SS_LEX) c[3] += sl.nbx;
    }
    for (int q = 0; q < 4; q++) sc[q][tid] = c[q];
    sact[tid] = act;
    __syncthreads();
    // inclusive Hillis-Steele scans
    for (int off = 1; off < 1024; off <<= 1) {
        int v[4], a = 0;
        for (int q = 0; q < 4; q++) v[q] = tid >= off ? sc[q][tid - off] : 0;
        if (tid >= off) a = sact[tid - off];
        __syncthreads();
        for (int q = 0; q < 4; q++) sc[q][tid] += v[q];
        sact[tid] += a;
        __syncthreads();
    }
    int o[4];
    for (int q = 0; q < 4; q++) o[q] = sc[q][tid] - c[q];
    int overflow = 0;
    for (int gid = g0; gid < g1; gid++) {
        int st = b.state[gid];
        if (st == SS_EMPTY || st == SS_DONE || b.held[gid / b.max_nt]) continue;
        const BSlot &sl = b.slots[gid / b.max_nt];
        if (st == SS_FP32 || st == SS_FP64 || st == SS_VERIFY) {
            int q = st == SS_FP32 ? 0 : 1;
            int2 *lst = q == 0 ? b.items32 : b.items64;
            for (int ch = 0; ch < sl.nbx; ch++, o[q]++)
                if (o[q] < b.cap_items) lst[o[q]] = make_int2(gid, ch);
                else overflow = 1;
        } else if (st == SS_PEND) {
            for (int ch = 0; ch < sl.nfull; ch++, o[2]++)
                if (o[2] < b.cap_pend) b.pend[o[2]] = make_int2(gid, ch);
                else overflow = 1;
        } else if (st == SS_LEX) {
            for (int ch = 0; ch < sl.nbx; ch++, o[3]++)
                if (o[3] < b.cap_pend) b.itemslex[o[3]] = make_int2(gid, ch);
                else overflow = 1;
        }
    }
    if (overflow) atomicOr(&b.counts[5], 1);
    if (tid == 1023) {
        b.counts[0] = min(sc[0][1023], b.cap_items);
        b.counts[1] = min(sc[1][1023], b.cap_items);
        b.counts[2] = min(sc[2][1023], b.cap_pend);
        b.counts[3] = sact[1023];
        b.counts[6] = 0;
        b.counts[7] = 0;
        b.counts[10] = min(sc[3][1023], b.cap_pend);
        for (int q = 11; q < 16; q++) b.counts[q] = 0;
    }
}

// ---------------------------------------------------------- the sweep kernels --
template <class S>
__device__ __forceinline__ void slot_fields(const BSlot &sl, typename S::V *&u, typename S::V *&g) {
    if constexpr (sizeof(typename S::T) == 8) {
        u = sl.u64r;
        g = sl.g64r;
    } else {
        u = sl.u32;
        g = sl.g32;
    }
}

// STG: the six links of a site are staged in shared memory by cp.async (dynamic
// shared memory of 6 x NS x BCHUNK x 16 bytes), as in the single-lattice kernel
template <class S, int MINB, bool STG>
__global__ void __launch_bounds__(BCHUNK, MINB) k_bsweep(BState b) {
    extern __shared__ __align__(16) unsigned char bstage[];
    using T = typename S::T;
    constexpr bool F64 = sizeof(T) == 8;
    __shared__ int next[2];
    const int n = b.counts[F64 ? 1 : 0];
    const int expect = F64 ? SS_FP64 : SS_FP32;
    const int2 *items = F64 ? b.items64 : b.items32;
    int *cursor = b.counts + (F64 ? 7 : 6);
    // the previous half-sweep's reunitarisation flags have been consumed
    if (!F64 && blockIdx.x == 0 && threadIdx.x == 0) b.counts[8] = b.counts[9] = b.counts[16] = 0;
    // Items come one at a time from a shared cursor, so a CTA held up by a
    // timeslice's final reduction does not hold back a fixed share of the list.
    // Thread 0 asks for item j + 1 while item j is processed and publishes it in
    // next[(j + 1) & 1] at the end of iteration j; that slot was last read in
    // iteration j - 1, before the barrier at the top of iteration j.
    if (threadIdx.x == 0) next[0] = atomicAdd(cursor, 1);
    for (int j = 0;; j++) {
        __syncthreads();
        const int it = next[j & 1];
        if (it >= n) break;
        int ahead = 0;
        if (threadIdx.x == 0) ahead = atomicAdd(cursor, 1);
        const int2 item = items[it];
        const int gid = item.x, chunk = item.y;
        // a timeslice retired earlier in this round still has items in the list;
        // the state is the same for every thread of the CTA
        const int st = *(volatile int *)&b.state[gid];
        const bool verify = F64 && st == SS_VERIFY;
        if (st == expect || verify) {
            // the same for every thread of the CTA: the parity of the timeslice's own
            // next half-sweep, and whether this pass measures e2
            const int par = b.sweeps[gid] & 1;
            const int track = verify ? 1 : (b.mflag[gid] & MF_NOW);
            const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
            const BSlot &sl = b.slots[slot];
            const Lat l = sl.l;   // a local copy: the stores below cannot be taken to change it
            typename S::V *u, *g;
            slot_fields<S>(sl, u, g);
            const uint32_t vsh = l.vs >> 1;
            const uint32_t off = (uint32_t)chunk * BCHUNK + threadIdx.x;
            double pre = 0.0, post = 0.0;
            if (off < vsh && verify) {
                pre = measure_site<S>(u, l, par, (uint32_t)t * vsh + off);
            } else if (off < vsh) {
                if constexpr (STG)
                    fast_site_staged<S, BCHUNK, false>(u, g, l, par, (uint32_t)t * vsh + off, (T)b.omega, b.hits,
                                                       track, pre, post, (typename S::V *)bstage);
                else
                    fast_site<S>(u, g, l, par, (uint32_t)t * vsh + off, (T)b.omega, b.hits, track, pre, post);
            }
            // the pieces' partials (warp w of the CTA sweeps piece w); k_bslice
            // combines them after the half-sweep
            if (track) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    pre += __shfl_down_sync(0xffffffffu, pre, o);
                    post += __shfl_down_sync(0xffffffffu, post, o);
                }
                if ((threadIdx.x & 31) == 0) {
                    double *pp = sl.part + (((size_t)t * sl.nbx + chunk) * BPIECES + (threadIdx.x >> 5)) * 2;
                    pp[0] = pre;
                    pp[1] = post;
                }
            }
        }
        if (threadIdx.x == 0) next[(j + 1) & 1] = ahead;
    }
}

// The same persistent half-sweep with one warp per CTA (the shape of the fastest
// single-lattice launches: 32-site blocks, 8-12 per SM).  A work item's BCHUNK sites
// are swept as BCHUNK / 32 pieces of 32, one after the other, each with its six
// links staged in shared memory (6 x NS x 32 x 16 B per CTA); a CTA never waits for
// the slowest of several warps, and the item's e2 partials are summed over its
// pieces per lane, then across the warp, in a fixed order.  Each thread stages into
// and reads back from its own shared-memory slots only, so no CTA barrier is needed.
// Pieces q0 .. q1 - 1 of a work item for k_bsweep_w / k_bsweep_wf (the whole item:
// 0 .. BPIECES), one after the other; each piece's e2 partials summed across the
// warp into the piece's own slot.
template <class S>
__device__ __forceinline__ void bsweep_pieces_w(const BState &b, int2 item, int q0, int q1, unsigned char *stage) {
    using T = typename S::T;
    constexpr bool F64 = sizeof(T) == 8;
    const int lane = threadIdx.x;
    const int expect = F64 ? SS_FP64 : SS_FP32;
    const int gid = item.x, chunk = item.y;
    const int st = *(volatile int *)&b.state[gid];
    const bool verify = F64 && st == SS_VERIFY;
    if (st != expect && !verify) return;   // retired earlier in this round (uniform)
    const int par = b.sweeps[gid] & 1;
    const int track = verify ? 1 : (b.mflag[gid] & MF_NOW);
    const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
    const BSlot &sl = b.slots[slot];
    // the geometry in registers: through a reference into the slot table the compiler
    // would read it again after every store of the update (it cannot rule out aliasing)
    const Lat l = sl.l;
    typename S::V *u, *g;
    slot_fields<S>(sl, u, g);
    const uint32_t vsh = l.vs >> 1;
#pragma unroll 1
    for (int q = q0; q < q1; q++) {
        const uint32_t off = (uint32_t)chunk * BCHUNK + (uint32_t)q * 32 + lane;
        double pre = 0.0, post = 0.0;
        if (off < vsh) {
            if (verify)
                pre = measure_site<S>(u, l, par, (uint32_t)t * vsh + off);
            else
                fast_site_staged<S, 32, false>(u, g, l, par, (uint32_t)t * vsh + off, (T)b.omega, b.hits, track, pre,
                                               post, (typename S::V *)stage);
        }
        if (track) {   // a piece past the end of the timeslice contributes zeros
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                pre += __shfl_down_sync(0xffffffffu, pre, o);
                post += __shfl_down_sync(0xffffffffu, post, o);
            }
            if (lane == 0) {
                double *pp = sl.part + (((size_t)t * sl.nbx + chunk) * BPIECES + q) * 2;
                pp[0] = pre;
                pp[1] = post;
            }
        }
    }
}

// The hand-out of a persistent half-sweep over n work items by gridDim.x CTAs: the
// first n - min(n, gridDim.x) items whole, then the last min(n, gridDim.x) items as
// 32-site pieces, so the CTAs finish within about a piece of one another (a lattice
// of few items fills the GPU too).  Cursor value c -> item, first and end piece.
struct Handout {
    int whole, end;   // items handed out whole; cursor values in use
    __device__ explicit Handout(int n) {
        const int tail = min(n, (int)gridDim.x);
        whole = n - tail;
        end = whole + tail * BPIECES;
    }
    __device__ int item(int c, int &q0, int &q1) const {
        if (c < whole) {
            q0 = 0;
            q1 = BPIECES;
            return c;
        }
        const int p = c - whole;
        q0 = p % BPIECES;
        q1 = q0 + 1;
        return whole + p / BPIECES;
    }
};

// Both precisions in one persistent launch of one-warp CTAs: the FP32 items first,
// then the FP64 ones, from one cursor, so a half-sweep has one tail instead of one
// per precision and one launch fewer.  A thread's staging slots are the same column
// of the shared array in both precisions' layouts.
template <int MINB>
__global__ void __launch_bounds__(32, MINB) k_bsweep_wf(BState b) {
    extern __shared__ __align__(16) unsigned char bstage[];
    const int n32 = b.counts[0];
    const Handout h(n32 + b.counts[1]);
    int *cursor = b.counts + 6;
    const int lane = threadIdx.x;
    // the previous half-sweep's reunitarisation flags have been consumed
    if (blockIdx.x == 0 && lane == 0) b.counts[8] = b.counts[9] = b.counts[16] = 0;
    int c = 0;
    if (lane == 0) c = atomicAdd(cursor, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    while (c < h.end) {
        // the next hand-out is requested while this one is swept
        int ahead = 0;
        if (lane == 0) ahead = atomicAdd(cursor, 1);
        int q0, q1;
        const int it = h.item(c, q0, q1);
        if (it < n32)
            bsweep_pieces_w<S32>(b, b.items32[it], q0, q1, bstage);
        else
            bsweep_pieces_w<S64R>(b, b.items64[it - n32], q0, q1, bstage);
        c = __shfl_sync(0xffffffffu, ahead, 0);
    }
}

template <class S, int MINB>
__global__ void __launch_bounds__(32, MINB) k_bsweep_w(BState b) {
    extern __shared__ __align__(16) unsigned char bstage[];
    constexpr bool F64 = sizeof(typename S::T) == 8;
    const Handout h(b.counts[F64 ? 1 : 0]);
    const int2 *items = F64 ? b.items64 : b.items32;
    int *cursor = b.counts + (F64 ? 7 : 6);
    const int lane = threadIdx.x;
    // the previous half-sweep's reunitarisation flags have been consumed
    if (!F64 && blockIdx.x == 0 && lane == 0) b.counts[8] = b.counts[9] = b.counts[16] = 0;
    int c = 0;
    if (lane == 0) c = atomicAdd(cursor, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    while (c < h.end) {
        int ahead = 0;
        if (lane == 0) ahead = atomicAdd(cursor, 1);
        int q0, q1;
        const int it = h.item(c, q0, q1);
        bsweep_pieces_w<S>(b, items[it], q0, q1, bstage);
        c = __shfl_sync(0xffffffffu, ahead, 0);
    }
}

// The k-th site of parity p of timeslice t in lexicographic order (odd ns): the
// timeslice's first row has row parity t & 1 (ns^2 is odd) and rows alternate, so a
// pair of rows holds exactly ns such sites; false past the last one.
__device__ __forceinline__ bool odd_parity_site_t(const Lat &l, int p, uint32_t t, uint32_t k, uint32_t &off) {
    const uint32_t ns = (uint32_t)l.ns;
    const uint32_t a = ((uint32_t)p ^ (t & 1u)) ? (ns - 1) >> 1 : (ns + 1) >> 1;
    const uint32_t pair = k / ns, rem = k - pair * ns;
    const uint32_t R = rem < a ? 2 * pair : 2 * pair + 1;
    const uint32_t j = rem < a ? rem : rem - a;
    const uint32_t x = 2 * j + ((uint32_t)p ^ ((R + t) & 1u));
    off = x + ns * R;
    return R < ns * ns;
}

// Odd-ns timeslices, boundary level `level` of one half-sweep: one-warp CTAs take
// 32-site pieces of the odd-ns work items (chunks of the timeslice's sites of the
// half-sweep's parity, numbered as above); a lane updates its site if it has the level.
// Sites of one level share no link, and every pair that does share one is in
// consecutive levels in the sequential sweep's order (see SS_LEX).
template <int MINB>
__global__ void __launch_bounds__(32, MINB) k_bsweep_lex(BState b, int level) {
    extern __shared__ __align__(16) unsigned char bstage[];
    const int n = b.counts[10] * BPIECES;
    int *cursor = b.counts + 11 + level;
    const int lane = threadIdx.x;
    int it = 0;
    if (lane == 0) it = atomicAdd(cursor, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    while (it < n) {
        int ahead = 0;
        if (lane == 0) ahead = atomicAdd(cursor, 1);
        const int2 item = b.itemslex[it / BPIECES];
        const int gid = item.x;
        // ns = 1: every spatial link closes on its own site and e2 vanishes identically,
        // so the fix leaves the lattice as it is (the half-sweeps pass it by until its
        // first e2 measurement retires it)
        if (*(volatile int *)&b.state[gid] == SS_LEX && b.slots[gid / b.max_nt].l.ns > 1) {   // uniform in the CTA
            const int par = b.sweeps[gid] & 1;
            const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
            const BSlot &sl = b.slots[slot];
            const Lat l = sl.l;
            // lanes take the sites of the half-sweep's parity only (k-th such site of
            // the timeslice); the pieces past the last one have nothing to do
            const uint32_t k = (uint32_t)item.y * BCHUNK + (uint32_t)(it % BPIECES) * 32 + lane;
            uint32_t off;
            if (odd_parity_site_t(l, par, (uint32_t)t, k, off)) {
                const uint32_t L = (uint32_t)t * l.vs + off;
                const Coord c = coord_lex(l, L);
                const uint32_t e = (uint32_t)l.ns - 1;
                const int lev = (int)(c.x == e) + (int)(c.y == e) + (int)(c.z == e);
                if (lev == level) {
                    double a = 0.0, z = 0.0;
                    fast_site_staged<S64R, 32, false, 6, false>(sl.u64r, sl.g64r, l, 0, L, b.omega, b.hits, 0, a, z,
                                                                 (double2 *)bstage);
                }
            }
        }
        it = __shfl_sync(0xffffffffu, ahead, 0);
    }
}

// e2 of the odd-ns timeslices measured on this half-sweep (mflag MF_NOW), over all
// their sites, on the state the four level launches left: one partial per piece.
__global__ void __launch_bounds__(32) k_bmeasure_lex(BState b) {
    const int n = b.counts[10];
    int *cursor = b.counts + 15;
    const int lane = threadIdx.x;
    int it = 0;
    if (lane == 0) it = atomicAdd(cursor, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    while (it < n) {
        int ahead = 0;
        if (lane == 0) ahead = atomicAdd(cursor, 1);
        const int2 item = b.itemslex[it];
        const int gid = item.x;
        if (*(volatile int *)&b.state[gid] == SS_LEX && (b.mflag[gid] & MF_NOW)) {   // uniform in the CTA
            const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
            const BSlot &sl = b.slots[slot];
            const Lat &l = sl.l;
#pragma unroll 1
            for (int q = 0; q < BPIECES; q++) {
                const uint32_t off = (uint32_t)item.y * BCHUNK + (uint32_t)q * 32 + lane;
                double v = off < l.vs ? measure_site<S64R, false>(sl.u64r, l, 0, (uint32_t)t * l.vs + off) : 0.0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) {
                    double *pp = sl.part + (((size_t)t * sl.nbx + item.y) * BPIECES + q) * 2;
                    pp[0] = v;
                    pp[1] = 0.0;
                }
            }
        }
        it = __shfl_sync(0xffffffffu, ahead, 0);
    }
}

// After both sweep kernels of a half-sweep, one warp per swept timeslice: advances its
// half-sweep count and e2 measurement schedule; where the half-sweep was measured,
// sums the chunk partials in a fixed order (lane-strided, then a shuffle tree) and,
// with the previous half-sweep measured too, has the timeslice's e2 after the
// previous half-sweep and retires it: FP32 -> pending switch at the switch
// threshold, FP64 -> done at the tolerance, NaN -> done with the status bit.
__global__ void k_bslice(BState b) {
    const int lane = threadIdx.x & 31;
    // both sweep kernels of this half-sweep have finished: count it and reset their
    // item cursors for the next one
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.counts[4] += 1;
        b.counts[6] = 0;
        b.counts[7] = 0;
        for (int q = 11; q < 16; q++) b.counts[q] = 0;
    }
    for (int gid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gid < b.nslices;
         gid += (gridDim.x * blockDim.x) >> 5) {
        const int st = b.state[gid];
        // swept in this half-sweep: listed at the round's start and not retired since
        // (a timeslice switched to FP64 at the start of the round has no items yet)
        if (!b.listed[gid] || (st != SS_FP32 && st != SS_FP64 && st != SS_VERIFY && st != SS_LEX))
            continue;   // uniform in the warp
        const int f = st == SS_VERIFY ? MF_NOW : b.mflag[gid];
        const int c = b.sweeps[gid];   // this half-sweep's own index
        const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
        const BSlot &sl = b.slots[slot];
        double s0 = 0.0, s1 = 0.0;
        if (f & MF_NOW) {
            const double *pp = sl.part + (size_t)t * sl.nbx * BPIECES * 2;
            for (int q = lane; q < sl.nbx * BPIECES; q += 32) {
                s0 += pp[2 * q];
                s1 += pp[2 * q + 1];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s0 += __shfl_down_sync(0xffffffffu, s0, o);
                s1 += __shfl_down_sync(0xffffffffu, s1, o);
            }
        }
        if (lane != 0) continue;
        if (st == SS_LEX) {
            // e2 of the state after this half-sweep, measured by k_bmeasure_lex
            int nf = f & MF_DENSE, nst = st;
            if (f & MF_NOW) {
                const double e2s = s0 / (double)sl.l.vs;
                if (!(s0 == s0)) {
                    atomicOr(b.status, GFC_STATUS_NAN);
                    nst = SS_DONE;
                } else if (e2s <= b.tol) {
                    nst = SS_DONE;
                } else if (!(nf & MF_DENSE)) {
                    if (e2s <= 1e3 * b.tol) {
                        nf |= MF_DENSE;
                    } else if (b.mk[gid] >= 0 && e2s < b.me2[gid]) {
                        const double rate = pow(e2s / b.me2[gid], 1.0 / (double)(c - b.mk[gid]));
                        if (e2s * pow(rate, 2.0 * MEASURE_PERIOD) <= 10.0 * b.tol) nf |= MF_DENSE;
                    }
                }
                b.mk[gid] = c;
                b.me2[gid] = e2s;
            }
            if ((nf & MF_DENSE) || measure_at(c + 1)) nf |= MF_NOW;
            b.mflag[gid] = nf;
            b.sweeps[gid] = c + 1;
            if (nst != st) b.state[gid] = nst;
            else if (b.reunit64 && (unsigned)(c + 1) % b.reunit64 == 0) b.counts[9] = 1;
            continue;
        }
        if (st == SS_VERIFY) {
            // measure-only pass: e2 of the current state = post of the last half-sweep
            // applied (index c - 1) + the other parity now; nothing was applied
            const double *rlast = b.ring + ((size_t)((c + 1) & 1) * b.nslices + gid) * 2;
            const double e2s = (s0 + rlast[1]) / (double)sl.l.vs;
            if (!(s0 == s0)) {
                atomicOr(b.status, GFC_STATUS_NAN);
                b.state[gid] = SS_DONE;
            } else if (e2s <= b.tol) {
                b.state[gid] = SS_DONE;
            } else {
                b.mflag[gid] = MF_NOW | MF_PREV | MF_DENSE;
                b.state[gid] = SS_FP64;
            }
            continue;
        }
        int nf = f & MF_DENSE;
        int nst = st;
        if (f & MF_NOW) {
            // ring by the timeslice's own half-sweep index: (pre, post) of c and c - 1
            double *rprev = b.ring + ((size_t)((c + 1) & 1) * b.nslices + gid) * 2;
            double *rcur = b.ring + ((size_t)(c & 1) * b.nslices + gid) * 2;
            rcur[0] = s0;
            rcur[1] = s1;
            if (!(s0 == s0) || !(s1 == s1)) {
                atomicOr(b.status, GFC_STATUS_NAN);
                nst = SS_DONE;
            } else if (f & MF_PREV) {
                const double e2s = (s0 + rprev[1]) / (double)sl.l.vs;   // e2 after half-sweep c - 1
                const double target = st == SS_FP32 ? b.switch_e2 : b.tol;
                if (e2s <= target) {
                    nst = st == SS_FP32 ? SS_PEND : SS_VERIFY;
                } else if (!(nf & MF_DENSE)) {
                    if (e2s <= 1e3 * target) {
                        nf |= MF_DENSE;
                    } else if (b.mk[gid] >= 0 && e2s < b.me2[gid]) {
                        const double rate = pow(e2s / b.me2[gid], 1.0 / (double)(c - 1 - b.mk[gid]));
                        if (e2s * pow(rate, 2.0 * MEASURE_PERIOD) <= 10.0 * target) nf |= MF_DENSE;
                    }
                }
                b.mk[gid] = c - 1;
                b.me2[gid] = e2s;
            }
            nf |= MF_PREV;
        }
        if ((nf & MF_DENSE) || measure_at(c + 1)) nf |= MF_NOW;
        // an FP32 rebuild after this half-sweep: the next measured pair must not
        // straddle it (its first half would see the links before the rebuild)
        const bool rebuild = nst == st && st == SS_FP32 && b.refresh32 && (unsigned)(c + 1) % b.refresh32 == 0;
        if (rebuild) {
            nf &= ~MF_PREV;
            b.counts[16] = 1;
        }
        b.mflag[gid] = nf;
        b.sweeps[gid] = c + 1;
        if (nst != st) {
            b.state[gid] = nst;
        } else {
            const unsigned period = st == SS_FP32 ? b.reunit32 : b.reunit64;
            if (period && (unsigned)(c + 1) % period == 0) b.counts[st == SS_FP32 ? 8 : 9] = 1;
        }
    }
}

// projectSU3 of a timeslice's working fields after every `period` of its own
// half-sweeps (its own count, so a lattice admitted later is treated exactly as if
// it were alone); the FP32 or the FP64 timeslices, by S
template <class S>
__device__ __forceinline__ void breunit_part(const BState &b, unsigned period, int *due, int &ndue,
                                             bool lex = false) {
    constexpr bool F64 = sizeof(typename S::T) == 8;
    if (period == 0 || !b.counts[F64 ? 9 : 8]) return;   // none is due this half-sweep (uniform)
    const int n = lex ? b.counts[10] : b.counts[F64 ? 1 : 0];
    const int2 *items = lex ? b.itemslex : (F64 ? b.items64 : b.items32);
    const int expect = lex ? SS_LEX : (F64 ? SS_FP64 : SS_FP32);
    // the CTA examines BCHUNK items at once (one per thread) and projects only the
    // chunks of timeslices that are due; most half-sweeps none are
    for (int base = blockIdx.x * BCHUNK; base < n; base += gridDim.x * BCHUNK) {
        if (threadIdx.x == 0) ndue = 0;
        __syncthreads();
        const int it = base + threadIdx.x;
        if (it < n) {
            const int gid = items[it].x;
            const int own = b.sweeps[gid];
            if (b.state[gid] == expect && own != 0 && (unsigned)own % period == 0) due[atomicAdd(&ndue, 1)] = it;
        }
        __syncthreads();
        for (int q = 0; q < ndue; q++) {   // independent chunks: their order does not matter
            const int2 item = items[due[q]];
            const int gid = item.x;
            const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
            const BSlot &sl = b.slots[slot];
            const Lat l = sl.l;
            typename S::V *u, *g;
            slot_fields<S>(sl, u, g);
            const uint32_t span = l.cb ? l.vs >> 1 : l.vs;   // sites of a timeslice per parity slot
            const uint32_t off = (uint32_t)item.y * BCHUNK + threadIdx.x;
            if (off >= span) continue;
            const uint32_t i = (uint32_t)t * span + off;
            for (int par = 0; par < l.npar; par++) {
                for (int d = 0; d <= 3; d++) {
                    typename S::V *p = d < 3 ? u + su_idx<S>(l, d, par, i) : g + sg_idx<S>(l, par, i);
                    Mt<typename S::T> m;
                    S::load(p, l.vh, m);
                    if (!fproject(m)) atomicOr(b.status, GFC_STATUS_PROJECT_FAIL);
                    S::store(p, l.vh, m);
                }
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(BCHUNK) k_breunit(BState b) {
    __shared__ int due[BCHUNK];
    __shared__ int ndue;
    breunit_part<S32>(b, b.reunit32, due, ndue);
    breunit_part<S64R>(b, b.reunit64, due, ndue);
    if (b.lex) breunit_part<S64R>(b, b.reunit64, due, ndue, true);
}

// ------------------------------------------------------ FP32 rebuilds --
// With options.fp32_refresh = K, an FP32 timeslice whose own half-sweep count reaches
// a multiple of K is rebuilt from FP64 (as the single-lattice mixed fix does): pass 1
// G <- Proj(Proj(G32) G) in FP64 and G32 back to the identity, pass 2 its FP32 links
// rounded from G(x) U0_d(x) G(x+d)^dagger computed in FP64 from the original links.
// Both passes return at once unless a rebuild is due this half-sweep; a CTA scans
// BCHUNK FP32 items at once and rebuilds the chunks of due timeslices only.
template <int PASS>
__global__ void __launch_bounds__(BCHUNK) k_brefresh(BState b) {
    __shared__ int due[BCHUNK];
    __shared__ int ndue;
    if (!b.refresh32 || !b.counts[16]) return;   // uniform
    const int n = b.counts[0];
    for (int base = blockIdx.x * BCHUNK; base < n; base += gridDim.x * BCHUNK) {
        if (threadIdx.x == 0) ndue = 0;
        __syncthreads();
        const int it = base + threadIdx.x;
        if (it < n) {
            const int gid = b.items32[it].x;
            const int own = b.sweeps[gid];
            if (b.state[gid] == SS_FP32 && own != 0 && (unsigned)own % b.refresh32 == 0)
                due[atomicAdd(&ndue, 1)] = it;
        }
        __syncthreads();
        for (int q = 0; q < ndue; q++) {   // independent chunks
            const int2 item = b.items32[due[q]];
            const int gid = item.x;
            const int slot = gid / b.max_nt, t = gid - slot * b.max_nt;
            const BSlot &sl = b.slots[slot];
            const Lat l = sl.l;
            const uint32_t span = l.vs >> 1;   // FP32 timeslices use the checkerboard layout
            const uint32_t off = (uint32_t)item.y * BCHUNK + threadIdx.x;
            if (off >= span) continue;
            const uint32_t i = (uint32_t)t * span + off;
            for (int par = 0; par < 2; par++) {
                if (PASS == 0) {
                    float4 *q32 = sl.g32 + sg_idx<S32>(l, par, i);
                    Mt<float> m32;
                    S32::load_rows01(q32, l.vh, m32);
                    Mt<double> m1, m0, r;
                    for (int e = 0; e < 6; e++) m1.e[e] = make_double2(m32.e[e].x, m32.e[e].y);
                    if (!fproject(m1)) fidentity(m1);
                    S64::load(sl.g + sg_idx<S64>(l, par, i), l.vh, m0);
                    fprod_left<S64, double>(m1, m0, r);
                    if (!fproject(r)) fidentity(r);
                    S64::store(sl.g + sg_idx<S64>(l, par, i), l.vh, r);
                    fidentity(m32);
                    S32::store(q32, l.vh, m32);
                } else {
                    const Coord c = coord_cb(l, par, i);
                    Mt<double> gx, gy, uu, tm, o;
                    S64::load(sl.g + sg_idx<S64>(l, par, i), l.vh, gx);
                    for (int d = 0; d < 3; d++) {
                        S64::load(sl.g + sg_idx<S64>(l, par ^ 1, fwd_L(l, c, d) >> 1), l.vh, gy);
                        S64::load(sl.u + uidx(l, d, par, 0, i), l.vh, uu);
                        fprod_left<S64R, double>(gx, uu, tm);
                        fprod_dag<S64R, double>(tm, gy, o);
                        Mt<float> of;
                        for (int e = 0; e < 6; e++) of.e[e] = make_float2((float)o.e[e].x, (float)o.e[e].y);
                        S32::store(sl.u32 + su_idx<S32>(l, d, par, i), l.vh, of);
                    }
                }
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------- FP32 -> FP64 switch --
// pass 1: G in FP64 (row 2 rebuilt from the FP32 rows, projected) into g and g64r
__global__ void __launch_bounds__(BCHUNK) k_switch_g(BState b) {
    const int n = b.counts[2];
    for (int it = blockIdx.x; it < n; it += gridDim.x) {
        const int2 item = b.pend[it];
        const int slot = item.x / b.max_nt, t = item.x - slot * b.max_nt;
        const BSlot &sl = b.slots[slot];
        const Lat l = sl.l;
        const uint32_t r = (uint32_t)item.y * BCHUNK + threadIdx.x;
        if (r >= l.vs) continue;
        const Slot s = slot_of(l, (uint32_t)t * l.vs + r);
        Mt<float> m32;
        S32::load_rows01(sl.g32 + sg_idx<S32>(l, s.par, s.i), l.vh, m32);
        Mt<double> m;
        for (int q = 0; q < 6; q++) m.e[q] = make_double2(m32.e[q].x, m32.e[q].y);
        if (!fproject(m)) fidentity(m);
        if (b.refresh32) {
            // composed with the G the rebuilds accumulated
            Mt<double> m0, r;
            S64::load(sl.g + sg_idx<S64>(l, s.par, s.i), l.vh, m0);
            fprod_left<S64, double>(m, m0, r);
            if (!fproject(r)) fidentity(r);
            m = r;
        }
        S64::store(sl.g + sg_idx<S64>(l, s.par, s.i), l.vh, m);
        S64R::store(sl.g64r + sg_idx<S64R>(l, s.par, s.i), l.vh, m);
    }
}

// pass 2: links U_d(x) = G(x) U0_d(x) G(x+d)^dagger from the FP64 originals into u64r
__global__ void __launch_bounds__(BCHUNK) k_switch_u(BState b) {
    const int n = b.counts[2];
    for (int it = blockIdx.x; it < n; it += gridDim.x) {
        const int2 item = b.pend[it];
        const int slot = item.x / b.max_nt, t = item.x - slot * b.max_nt;
        const BSlot &sl = b.slots[slot];
        const Lat l = sl.l;
        const uint32_t r = (uint32_t)item.y * BCHUNK + threadIdx.x;
        if (r >= l.vs) continue;
        const uint32_t L = (uint32_t)t * l.vs + r;
        const Coord c = coord_lex(l, L);
        const Slot s = slot_of(l, L);
        M3 gx;
        load_m(sl.g + gidx(l, s.par, 0, s.i), l.vh, gx);
        for (int d = 0; d < 3; d++) {
            const Slot sy = slot_of(l, fwd_L(l, c, d));
            M3 gy, u0, tmp, o;
            load_m(sl.g + gidx(l, sy.par, 0, sy.i), l.vh, gy);
            load_m(sl.u + uidx(l, d, s.par, 0, s.i), l.vh, u0);
            xprod(gx, u0, tmp);
            xprod_dag(tmp, gy, o);
            double2 *q = sl.u64r + su_idx<S64R>(l, d, s.par, s.i);
#pragma unroll
            for (int e = 0; e < 6; e++) q[(size_t)e * l.vh] = o.e[e];
        }
    }
}

// pass 3: pending timeslices become FP64; the previous e2 entry is invalidated
__global__ void k_switch_done(BState b) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= b.nslices || b.state[gid] != SS_PEND) return;
    b.state[gid] = SS_FP64;
    b.ring[((size_t)0 * b.nslices + gid) * 2 + 1] = __longlong_as_double(0x7ff0000000000000LL);
    b.ring[((size_t)1 * b.nslices + gid) * 2 + 1] = __longlong_as_double(0x7ff0000000000000LL);
    b.mflag[gid] = measure_at(b.sweeps[gid]) ? MF_NOW : 0;   // a new target: measure afresh
    b.mk[gid] = -1;
}

// activate the timeslices of one slot in `state`
__global__ void k_activate(BState b, int gid0, int nt, int state) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int gid = gid0 + t;
    b.state[gid] = state;
    b.sweeps[gid] = 0;
    b.mflag[gid] = measure_at(0) ? MF_NOW : 0;
    b.mk[gid] = -1;
    for (int q = 0; q < 2; q++) {
        b.ring[((size_t)q * b.nslices + gid) * 2] = 0.0;
        b.ring[((size_t)q * b.nslices + gid) * 2 + 1] = __longlong_as_double(0x7ff0000000000000LL);
    }
}

__global__ void k_set_state(int *state, int gid0, int nt, int value) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nt) state[gid0 + t] = value;
}

}  // namespace gfc

using namespace gfc;

// ================================================================== host ==
struct gfc_batch {
    int dev = 0;
    cudaStream_t s = nullptr;
    int max_slots = 0, max_nt = 0, nslices = 0;
    size_t max_sites = 0, used_sites = 0;
    std::vector<BSlot> hs;          // host copies of the descriptors
    std::vector<void *> mem;        // per-slot allocation
    std::vector<int> used, ns, nt, activated, hheld;
    int *held = nullptr;            // device copy of hheld
    BSlot *dslots = nullptr;
    int *state = nullptr, *sweeps = nullptr, *counts = nullptr, *listed = nullptr, *mflag = nullptr, *mk = nullptr;
    double *me2 = nullptr;
    double *ring = nullptr;
    int2 *items32 = nullptr, *items64 = nullptr, *pend = nullptr, *itemslex = nullptr;
    int cap_items = 0, cap_pend = 0;
    int odd_slots = 0;               // slots of odd ns in use (their launches join the round)
    unsigned *status = nullptr;
    int *hcounts = nullptr;          // pinned mirror [8]
    int *hstate = nullptr;           // pinned mirror [nslices]
    // observables scratch (sized for the largest slot)
    double *part = nullptr, *dres = nullptr, *hres = nullptr;
    size_t part_n = 0;
    // the captured round
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int round_k = 8;
    BState captured{};
    int grid = 0, nsm = 0;
    int minb32 = 12, minb64 = 12, stage64 = 1;   // one-warp CTAs, 12 per SM (measured fastest on a mix)
    // slot memory: a pool of its own that keeps freed memory mapped, so a slot
    // freed and another admitted costs no unmapping and remapping of device memory
    cudaMemPool_t pool = nullptr;
    long long launches = 0;
    long long rounds = 0;
};

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

extern "C" int gfc_batch_create(int device, size_t max_sites, int max_slots, int max_nt, gfc_batch **out) {
    if (!out || max_slots <= 0 || max_nt <= 0 || max_sites == 0) return GFC_ERR_ARG;
    *out = nullptr;
    gfc_batch *b = new gfc_batch();
    b->dev = device;
    b->max_slots = max_slots;
    b->max_nt = max_nt;
    b->nslices = max_slots * max_nt;
    b->max_sites = max_sites;
    b->hs.assign(max_slots, BSlot{});
    b->mem.assign(max_slots, nullptr);
    b->used.assign(max_slots, 0);
    b->ns.assign(max_slots, 0);
    b->nt.assign(max_slots, 0);
    b->activated.assign(max_slots, 0);
    b->hheld.assign(max_slots, 0);
    // work lists: every chunk of every timeslice (upper bound)
    b->cap_items = (int)(max_sites / 2 / BCHUNK + (size_t)b->nslices + 1024);
    b->cap_pend = (int)(max_sites / BCHUNK + (size_t)b->nslices + 1024);
    int rc = GFC_OK;
    cudaError_t e;
#define BTRY(call)                          \
    if ((e = (call)) != cudaSuccess) {      \
        rc = cuda_fail(e, #call);           \
        goto fail;                          \
    }
    BTRY(cudaSetDevice(device));
    BTRY(cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking));
    BTRY(cudaMalloc(&b->dslots, sizeof(BSlot) * max_slots));
    BTRY(cudaMemset(b->dslots, 0, sizeof(BSlot) * max_slots));
    BTRY(cudaMalloc(&b->state, sizeof(int) * b->nslices));
    BTRY(cudaMemset(b->state, 0, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->sweeps, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->held, sizeof(int) * max_slots));
    BTRY(cudaMemset(b->held, 0, sizeof(int) * max_slots));
    BTRY(cudaMalloc(&b->listed, sizeof(int) * b->nslices));
    BTRY(cudaMemset(b->listed, 0, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->mflag, sizeof(int) * b->nslices));
    BTRY(cudaMemset(b->mflag, 0, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->mk, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->me2, sizeof(double) * b->nslices));
    BTRY(cudaMemset(b->sweeps, 0, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->ring, sizeof(double) * 4 * b->nslices));
    BTRY(cudaMalloc(&b->items32, sizeof(int2) * b->cap_items));
    BTRY(cudaMalloc(&b->items64, sizeof(int2) * b->cap_items));
    BTRY(cudaMalloc(&b->pend, sizeof(int2) * b->cap_pend));
    BTRY(cudaMalloc(&b->itemslex, sizeof(int2) * b->cap_pend));   // chunks over whole timeslices
    BTRY(cudaMalloc(&b->counts, sizeof(int) * 17));
    BTRY(cudaMemset(b->counts, 0, sizeof(int) * 17));
    BTRY(cudaMalloc(&b->status, sizeof(unsigned)));
    BTRY(cudaMemset(b->status, 0, sizeof(unsigned)));
    BTRY(cudaMallocHost(&b->hcounts, sizeof(int) * 8));
    BTRY(cudaMallocHost(&b->hstate, sizeof(int) * b->nslices));
    BTRY(cudaMalloc(&b->dres, sizeof(double) * 8));
    {
        cudaMemPoolProps pp{};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        BTRY(cudaMemPoolCreate(&b->pool, &pp));
        uint64_t keep = UINT64_MAX;
        BTRY(cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    BTRY(cudaMallocHost(&b->hres, sizeof(double) * 8));
    {
        int nsm = 0;
        BTRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        b->nsm = nsm;
        b->grid = nsm * 4;   // persistent CTAs of the reunit / switch kernels (they loop)
    }
#undef BTRY
    *out = b;
    return GFC_OK;
fail:
    delete b;
    return rc;
}

extern "C" int gfc_batch_destroy(gfc_batch *b) {
    if (!b) return GFC_ERR_ARG;
    cudaSetDevice(b->dev);
    cudaStreamSynchronize(b->s);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void *m : b->mem)
        if (m) cudaFreeAsync(m, b->s);
    cudaStreamSynchronize(b->s);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    cudaFree(b->dslots);
    cudaFree(b->state);
    cudaFree(b->sweeps);
    cudaFree(b->listed);
    cudaFree(b->held);
    cudaFree(b->mflag);
    cudaFree(b->mk);
    cudaFree(b->me2);
    cudaFree(b->ring);
    cudaFree(b->items32);
    cudaFree(b->items64);
    cudaFree(b->pend);
    cudaFree(b->itemslex);
    cudaFree(b->counts);
    cudaFree(b->status);
    cudaFree(b->part);
    cudaFree(b->dres);
    cudaFreeHost(b->hcounts);
    cudaFreeHost(b->hstate);
    cudaFreeHost(b->hres);
    if (b->s) cudaStreamDestroy(b->s);
    delete b;
    return GFC_OK;
}

// bytes of device memory one slot of ns^3 x nt needs
// chunks of one timeslice's sites of one parity slot (odd ns: the whole timeslice)
static size_t slot_chunks(const Lat &l) { return ((l.cb ? l.vs >> 1 : l.vs) + BCHUNK - 1) / BCHUNK; }

extern "C" size_t gfc_batch_slot_bytes(int ns, int nt) {
    Lat l = make_lat(ns, nt);
    const size_t m = (size_t)l.npar * l.vh;   // matrices per field (V)
    const size_t nbx = slot_chunks(l);
    return al256(3 * m * 9 * 16) + 2 * al256(m * 9 * 16)            // u, ut, g
           + al256(3 * m * 6 * 16) + al256(m * 6 * 16)              // u64r, g64r
           + al256(3 * m * 3 * 16) + al256(m * 3 * 16)              // u32, g32
           + al256((size_t)nt * nbx * BPIECES * 2 * 8) + 4096;      // piece partials
}

extern "C" int gfc_batch_add(gfc_batch *b, int ns, int nt, int *slot_out) {
    if (!b || !slot_out) return GFC_ERR_ARG;
    *slot_out = -1;
    if (ns <= 0 || nt <= 0 || nt > b->max_nt) {
        set_error("batch slots need ns > 0 and 0 < nt <= %d (got %d, %d)", b->max_nt, ns, nt);
        return GFC_ERR_GEOMETRY;
    }
    const size_t V = (size_t)ns * ns * ns * nt;
    if (V * 4 >= (1ull << 31)) return GFC_ERR_GEOMETRY;
    if (b->used_sites + V > b->max_sites) {
        set_error("batch capacity: %zu sites in use, %zu requested, %zu maximum", b->used_sites, V, b->max_sites);
        return GFC_ERR_BUSY;
    }
    int slot = -1;
    for (int k = 0; k < b->max_slots; k++)
        if (!b->used[k]) {
            slot = k;
            break;
        }
    if (slot < 0) {
        set_error("batch has no free slot (%d in use)", b->max_slots);
        return GFC_ERR_BUSY;
    }
    GFC_CHECK(cudaSetDevice(b->dev));
    const size_t bytes = gfc_batch_slot_bytes(ns, nt);
    void *m = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&m, bytes, b->pool, b->s);
    if (e != cudaSuccess) {
        // memory kept by the pool may be split badly for this size: return it and retry
        cudaGetLastError();
        GFC_CHECK(cudaStreamSynchronize(b->s));
        GFC_CHECK(cudaMemPoolTrimTo(b->pool, 0));
        e = cudaMallocFromPoolAsync(&m, bytes, b->pool, b->s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device memory for a %d^3x%d slot (%zu bytes): %s", ns, nt, bytes, cudaGetErrorString(e));
        return GFC_ERR_NOMEM;
    }
    BSlot sl{};
    sl.l = make_lat(ns, nt);
    const size_t mv = (size_t)sl.l.npar * sl.l.vh;   // matrices per field (V)
    char *p = (char *)m;
    auto take = [&](size_t n) {
        char *q = p;
        p += al256(n);
        return q;
    };
    sl.u = (double2 *)take(3 * mv * 9 * 16);
    sl.ut = (double2 *)take(mv * 9 * 16);
    sl.g = (double2 *)take(mv * 9 * 16);
    sl.u64r = (double2 *)take(3 * mv * 6 * 16);
    sl.g64r = (double2 *)take(mv * 6 * 16);
    sl.u32 = (float4 *)take(3 * mv * 3 * 16);
    sl.g32 = (float4 *)take(mv * 3 * 16);
    sl.nbx = (int)slot_chunks(sl.l);
    sl.nfull = (int)((sl.l.vs + BCHUNK - 1) / BCHUNK);
    sl.part = (double *)take((size_t)nt * sl.nbx * BPIECES * 2 * 8);
    GFC_CHECK(cudaMemcpyAsync(b->dslots + slot, &sl, sizeof sl, cudaMemcpyHostToDevice, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));   // the host copy of sl goes out of scope
    b->hs[slot] = sl;
    b->mem[slot] = m;
    b->used[slot] = 1;
    b->activated[slot] = 0;
    if (b->hheld[slot]) {
        b->hheld[slot] = 0;
        GFC_CHECK(cudaMemcpyAsync(b->held + slot, &b->hheld[slot], sizeof(int), cudaMemcpyHostToDevice, b->s));
        GFC_CHECK(cudaStreamSynchronize(b->s));
    }
    b->ns[slot] = ns;
    b->nt[slot] = nt;
    b->used_sites += V;
    b->odd_slots += ns & 1;
    // observables scratch large enough for every slot seen so far
    size_t need = (size_t)nt * obs_blocks_per_slice(sl.l) * 4;
    if (need > b->part_n) {
        cudaFree(b->part);
        b->part = nullptr;
        GFC_CHECK(cudaMalloc(&b->part, need * sizeof(double)));
        b->part_n = need;
    }
    *slot_out = slot;
    return GFC_OK;
}

// Keep a slot resident but out of the next rounds (hold != 0), or let it sweep again.
// Its timeslices keep their state, counts and measurements, so holding a lattice for
// some rounds changes when it finishes, not what it computes.
extern "C" int gfc_batch_hold(gfc_batch *b, int slot, int hold) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot]) return GFC_ERR_ARG;
    const int v = hold != 0;
    if (b->hheld[slot] == v) return GFC_OK;
    GFC_CHECK(cudaSetDevice(b->dev));
    b->hheld[slot] = v;
    GFC_CHECK(cudaMemcpyAsync(b->held + slot, &b->hheld[slot], sizeof(int), cudaMemcpyHostToDevice, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    return GFC_OK;
}

extern "C" int gfc_batch_remove(gfc_batch *b, int slot) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot]) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    GFC_CHECK(cudaMemsetAsync(b->state + (size_t)slot * b->max_nt, 0, sizeof(int) * b->max_nt, b->s));
    BSlot empty{};
    GFC_CHECK(cudaMemcpyAsync(b->dslots + slot, &empty, sizeof empty, cudaMemcpyHostToDevice, b->s));
    GFC_CHECK(cudaFreeAsync(b->mem[slot], b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    b->mem[slot] = nullptr;
    b->used[slot] = 0;
    b->used_sites -= (size_t)b->ns[slot] * b->ns[slot] * b->ns[slot] * b->nt[slot];
    b->odd_slots -= b->ns[slot] & 1;
    b->hs[slot] = BSlot{};
    return GFC_OK;
}

static int check_slot(gfc_batch *b, int slot) {
    if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot]) return GFC_ERR_ARG;
    return GFC_OK;
}

// Host links (reference layout, raw file bytes) into the slot, then reunitarised.
extern "C" int gfc_batch_upload(gfc_batch *b, int slot, const void *host, int elem_bytes, int byteswap) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    if (!host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    const Lat &l = sl.l;
    // stage through the slot's two-row FP64 field (not live before activation)
    const size_t per_slice = (size_t)l.vs * 4 * 18 * elem_bytes;
    // the working copies (u64r .. g32, contiguous) are dead outside a fix: >= 576 B per site
    const size_t stage = (size_t)((char *)sl.part - (char *)sl.u64r);
    const uint32_t per = (uint32_t)std::max<size_t>(1, stage / per_slice);
    for (uint32_t t0 = 0; t0 < (uint32_t)l.nt; t0 += per) {
        uint32_t n = std::min<uint32_t>(per, l.nt - t0);
        GFC_CHECK(cudaMemcpyAsync(sl.u64r, (const char *)host + (size_t)t0 * per_slice, n * per_slice,
                                  cudaMemcpyHostToDevice, b->s));
        // byte swap, precision, layout and reunitarisation in one pass
        launch_load_links(sl.u64r, elem_bytes, byteswap, l, t0, n, sl.u, sl.ut, b->s, 1, b->status);
    }
    b->launches += (l.nt + per - 1) / per;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

// The seeded synthetic configuration built on the device, then reunitarised.
extern "C" int gfc_batch_synth(gfc_batch *b, int slot, uint64_t seed, double scale) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    launch_synth(sl.l, seed, scale, sl.g, sl.u, sl.ut, b->s);
    launch_reunitarize(sl.u, sl.l.vh, 3 * sl.l.npar, b->status, b->s);
    launch_reunitarize(sl.ut, sl.l.vh, sl.l.npar, b->status, b->s);
    b->launches += 4;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

// G = 1 and the working copies for the first round; precision GFC_PREC_MIXED
// starts in FP32, anything else starts in FP64.
extern "C" int gfc_batch_activate(gfc_batch *b, int slot, int precision) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    const Lat &l = sl.l;
    launch_identity(sl.g, l, b->s);
    int st;
    if (!l.cb) {
        // odd ns: FP64 on two stored rows in the lexicographic layout, whatever the
        // precision asked for (the FP32 phase and its switch need the checkerboard)
        launch_pack2(sl.u, sl.u64r, l.vh, 3 * l.npar, b->s);
        launch_pack2(sl.g, sl.g64r, l.vh, l.npar, b->s);
        st = SS_LEX;
    } else if (precision == GFC_PREC_MIXED) {
        launch_to_f32(sl.u, sl.u32, l.vh, 3 * l.npar, b->s);
        launch_identity32(sl.g32, l.vh, l.npar, b->s);
        st = SS_FP32;
    } else {
        launch_pack2(sl.u, sl.u64r, l.vh, 3 * l.npar, b->s);
        launch_pack2(sl.g, sl.g64r, l.vh, l.npar, b->s);
        st = SS_FP64;
    }
    BState bs{};
    bs.nslices = b->nslices;
    bs.state = b->state;
    bs.sweeps = b->sweeps;
    bs.ring = b->ring;
    bs.mflag = b->mflag;
    bs.mk = b->mk;
    k_activate<<<(l.nt + 127) / 128, 128, 0, b->s>>>(bs, slot * b->max_nt, l.nt, st);
    b->launches += 5;
    b->activated[slot] = 1;
    GFC_CHECK(cudaGetLastError());
    return GFC_OK;
}

static BState make_state(gfc_batch *b, const gfc_params *p, const gfc_options *o) {
    BState s;
    memset(&s, 0, sizeof s);   // padding too: captured parameters are compared bytewise
    s.slots = b->dslots;
    s.max_nt = b->max_nt;
    s.nslices = b->nslices;
    s.state = b->state;
    s.sweeps = b->sweeps;
    s.listed = b->listed;
    s.held = b->held;
    s.mflag = b->mflag;
    s.mk = b->mk;
    s.me2 = b->me2;
    s.ring = b->ring;
    s.items32 = b->items32;
    s.items64 = b->items64;
    s.itemslex = b->itemslex;
    s.lex = b->odd_slots > 0;
    s.pend = b->pend;
    s.cap_items = b->cap_items;
    s.cap_pend = b->cap_pend;
    s.counts = b->counts;
    s.status = b->status;
    s.omega = (double)p->omega_OR;
    s.hits = p->hits;
    const double tol = p->gfix_proxy == GFC_PROXY_THETA ? 6.0 * p->tolerance : p->tolerance;
    s.tol = tol;
    s.switch_e2 = std::max(o->switch_e2 > 0 ? o->switch_e2 : 1e-9, tol);
    s.reunit64 = o->refine_reunit ? o->refine_reunit : p->sweeps_to_reunitarization;
    s.refresh32 = o->fp32_refresh > 0 ? (unsigned)o->fp32_refresh : 0u;
    // a rebuild takes the FP32 reunitarisation's place
    s.reunit32 = s.refresh32 ? 0u : std::min<unsigned>(p->sweeps_to_reunitarization, 50u);
    return s;
}

template <class S, int MINB, bool STG>
static void launch_bsweep_k(int grid, cudaStream_t st, const BState &bs) {
    constexpr size_t bytes = STG ? (size_t)6 * S::NS * BCHUNK * 16 : 0;
    auto kern = k_bsweep<S, MINB, STG>;
    if constexpr (STG) {
        static std::atomic<unsigned long long> done{0};
        smem_attr_once(done, kern, bytes);
    }
    kern<<<grid, BCHUNK, bytes, st>>>(bs);
}

static void launch_bsweep_lex(int grid, cudaStream_t st, const BState &bs, int level) {
    constexpr size_t bytes = (size_t)6 * S64R::NS * 32 * 16;
    auto kern = k_bsweep_lex<11>;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, kern, bytes);
    kern<<<grid, 32, bytes, st>>>(bs, level);
}

template <int MINB>
static void launch_bsweep_wf_k(int grid, cudaStream_t st, const BState &bs) {
    constexpr size_t bytes = (size_t)6 * S64R::NS * 32 * 16;   // the larger of the two layouts
    auto kern = k_bsweep_wf<MINB>;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, kern, bytes);
    kern<<<grid, 32, bytes, st>>>(bs);
}

// both precisions in one launch of one-warp CTAs, minb (8, 11 or 12) per SM
static void launch_bsweep_fused(int minb, int grid, cudaStream_t st, const BState &bs) {
    switch (minb) {
        case 8: return launch_bsweep_wf_k<8>(grid, st, bs);
        case 12: return launch_bsweep_wf_k<12>(grid, st, bs);
        default: return launch_bsweep_wf_k<11>(grid, st, bs);
    }
}

template <class S, int MINB>
static void launch_bsweep_w(int grid, cudaStream_t st, const BState &bs) {
    constexpr size_t bytes = (size_t)6 * S::NS * 32 * 16;
    auto kern = k_bsweep_w<S, MINB>;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once(done, kern, bytes);
    kern<<<grid, 32, bytes, st>>>(bs);
}

// minb: minimum resident CTAs per SM: 1..4 CTAs of BCHUNK threads (stage: FP64 links
// staged in shared memory, two-row FP64 only; 72 KiB per CTA, so at most 3 CTAs per
// SM), or 8, 11 or 12 one-warp CTAs with staged links (k_bsweep_w)
template <class S>
static void launch_bsweep(int minb, bool stage, int grid, cudaStream_t st, const BState &bs) {
    switch (minb) {
        case 8: return launch_bsweep_w<S, 8>(grid, st, bs);
        case 11: return launch_bsweep_w<S, 11>(grid, st, bs);
        case 12: return launch_bsweep_w<S, 12>(grid, st, bs);
        default: break;
    }
    if constexpr (sizeof(typename S::T) == 8) {
        if (stage) {
            switch (minb) {
                case 1: return launch_bsweep_k<S, 1, true>(grid, st, bs);
                case 2: return launch_bsweep_k<S, 2, true>(grid, st, bs);
                default: return launch_bsweep_k<S, 3, true>(grid, st, bs);
            }
        }
    }
    switch (minb) {
        case 1: return launch_bsweep_k<S, 1, false>(grid, st, bs);
        case 2: return launch_bsweep_k<S, 2, false>(grid, st, bs);
        case 3: return launch_bsweep_k<S, 3, false>(grid, st, bs);
        default: return launch_bsweep_k<S, 4, false>(grid, st, bs);
    }
}

// enqueue one round on the stream (used for capture)
static void enqueue_round(gfc_batch *b, const BState &bs) {
    cudaStream_t st = b->s;
    k_compact<<<1, 1024, 0, st>>>(bs);
    k_switch_g<<<b->grid, BCHUNK, 0, st>>>(bs);
    k_switch_u<<<b->grid, BCHUNK, 0, st>>>(bs);
    k_switch_done<<<(b->nslices + 255) / 256, 256, 0, st>>>(bs);
    for (int k = 0; k < b->round_k; k++) {
        // one resident wave of persistent CTAs: a CTA that had to wait for a slot
        // would start its share of the items late and stretch the tail
        if (b->minb32 > 4 && b->minb64 > 4) {
            // one-warp CTAs for both precisions: one launch, the FP64 shape
            launch_bsweep_fused(b->minb64, b->nsm * b->minb64, st, bs);
        } else {
            const int m64 = b->stage64 && b->minb64 <= 4 ? std::min(b->minb64, 3) : b->minb64;
            launch_bsweep<S32>(b->minb32, false, b->nsm * b->minb32, st, bs);
            launch_bsweep<S64R>(m64, b->stage64 != 0, b->nsm * m64, st, bs);
        }
        if (bs.lex) {
            // odd-ns timeslices: the four boundary levels in order, then their e2
            for (int level = 0; level < 4; level++) launch_bsweep_lex(b->nsm * 11, st, bs, level);
            k_bmeasure_lex<<<b->nsm * 16, 32, 0, st>>>(bs);
        }
        k_bslice<<<(b->nslices + 7) / 8, 256, 0, st>>>(bs);
        k_breunit<<<b->grid, BCHUNK, 0, st>>>(bs);
        if (bs.refresh32) {
            k_brefresh<0><<<b->grid, BCHUNK, 0, st>>>(bs);
            k_brefresh<1><<<b->grid, BCHUNK, 0, st>>>(bs);
        }
    }
}

static int ensure_graph(gfc_batch *b, const gfc_params *p, const gfc_options *o) {
    BState bs = make_state(b, p, o);
    if (b->exec && !memcmp(&bs, &b->captured, sizeof bs)) return GFC_OK;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    GFC_CHECK(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    enqueue_round(b, bs);
    GFC_CHECK(cudaStreamEndCapture(b->s, &b->graph));
    GFC_CHECK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->captured = bs;
    return GFC_OK;
}

// One round (K half-sweeps of every active timeslice).  *active = timeslices still
// working after it; the state table is copied back for gfc_batch_slot_status.
extern "C" int gfc_batch_round(gfc_batch *b, const gfc_params *p, const gfc_options *o, int *active) {
    if (!b || !p) return GFC_ERR_ARG;
    gfc_options od;
    if (!o) {
        gfc_options_default(&od);
        od.precision = GFC_PREC_MIXED;
        o = &od;
    }
    GFC_CHECK(cudaSetDevice(b->dev));
    int rc = ensure_graph(b, p, o);
    if (rc) return rc;
    GFC_CHECK(cudaGraphLaunch(b->exec, b->s));
    b->launches += 4 + ((b->minb32 > 4 && b->minb64 > 4 ? 3 : 4) + (b->odd_slots > 0 ? 5 : 0) +
                        (o->fp32_refresh > 0 ? 2 : 0)) * b->round_k;
    b->rounds++;
    GFC_CHECK(cudaMemcpyAsync(b->hcounts, b->counts, sizeof(int) * 8, cudaMemcpyDeviceToHost, b->s));
    GFC_CHECK(cudaMemcpyAsync(b->hstate, b->state, sizeof(int) * b->nslices, cudaMemcpyDeviceToHost, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    if (b->hcounts[5]) {
        set_error("batch work list overflow");
        return GFC_ERR_STATE;
    }
    // active timeslices after the round (the count in hcounts[3] is from its start)
    int act = 0;
    for (int g = 0; g < b->nslices; g++) act += b->hstate[g] != SS_EMPTY && b->hstate[g] != SS_DONE;
    if (active) *active = act;
    return GFC_OK;
}

// 1 if every timeslice of the slot has retired (from the state copied by the last round)
extern "C" int gfc_batch_slot_done(gfc_batch *b, int slot, int *done) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    if (!done) return GFC_ERR_ARG;
    int d = b->activated[slot];
    for (int t = 0; t < b->nt[slot] && d; t++) d = b->hstate[(size_t)slot * b->max_nt + t] == SS_DONE;
    *done = d;
    return GFC_OK;
}

// After retirement: canonical FP64 links and G, reunitarised; temporal links
// transformed; report with the largest per-timeslice half-sweep count and the
// observables of the fixed lattice.
extern "C" int gfc_batch_finalize(gfc_batch *b, int slot, gfc_report *r) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    const Lat &l = sl.l;
    k_set_state<<<(l.nt + 127) / 128, 128, 0, b->s>>>(b->state, slot * b->max_nt, l.nt, SS_DONE);
    launch_unpack2(sl.u64r, sl.u, l.vh, 3 * l.npar, b->s);
    launch_unpack2(sl.g64r, sl.g, l.vh, l.npar, b->s);
    launch_reunitarize(sl.u, l.vh, 3 * l.npar, b->status, b->s);
    launch_reunitarize(sl.g, l.vh, l.npar, b->status, b->s);
    launch_temporal_transform(sl.ut, sl.g, l, b->s);
    launch_reunitarize(sl.ut, l.vh, l.npar, b->status, b->s);
    b->launches += 6;
    if (r) {
        memset(r, 0, sizeof *r);
        std::vector<int> sw(l.nt);
        GFC_CHECK(cudaMemcpyAsync(sw.data(), b->sweeps + (size_t)slot * b->max_nt, sizeof(int) * l.nt,
                                  cudaMemcpyDeviceToHost, b->s));
        launch_obs(sl.u, l, b->part, b->dres, nullptr, b->s);
        launch_functional(sl.u, l, b->part, b->dres + 2, b->s);
        b->launches += 4;
        GFC_CHECK(cudaMemcpyAsync(b->hres, b->dres, sizeof(double) * 3, cudaMemcpyDeviceToHost, b->s));
        GFC_CHECK(cudaStreamSynchronize(b->s));
        int mx = 0;
        long long tot = 0;
        for (int t = 0; t < l.nt; t++) {
            mx = std::max(mx, sw[t]);
            tot += sw[t];
        }
        r->sweeps = mx;
        r->site_updates = tot * (long long)(l.vs / 2);
        r->e2 = b->hres[0] / (double)l.v;
        r->theta = b->hres[1] / (3.0 * (double)l.v);
        r->functional = b->hres[2] / ((double)l.v * 9.0);
        r->final_residue = r->e2;
        r->status = mx;
    } else {
        GFC_CHECK(cudaStreamSynchronize(b->s));   // a copy on another stream may follow
    }
    GFC_CHECK(cudaGetLastError());
    b->activated[slot] = 0;
    return GFC_OK;
}

extern "C" int gfc_batch_plaquette(gfc_batch *b, int slot, double *spatial, double *temporal) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    launch_plaquette(sl.u, sl.ut, sl.l, b->part, b->dres, b->s);
    GFC_CHECK(cudaMemcpyAsync(b->hres, b->dres, sizeof(double) * 2, cudaMemcpyDeviceToHost, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    if (spatial) *spatial = b->hres[0] / (3.0 * (double)sl.l.v);
    if (temporal) *temporal = b->hres[1] / (3.0 * (double)sl.l.v);
    return GFC_OK;
}

namespace gfc {
// G of a finalised slot to host memory on stream `st` (the caller's stream: the
// request server downloads on its own stream while rounds run on the batch's)
int batch_download_gt_on(gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap, cudaStream_t st) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    if (b->activated[slot]) {
        set_error("slot %d is still being fixed (finalize it first)", slot);
        return GFC_ERR_STATE;
    }
    if (!host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    const Lat &l = sl.l;
    // raw output staged through the (dead) FP64 two-row field
    const size_t per_slice = (size_t)l.vs * 18 * elem_bytes;
    // the working copies (u64r .. g32, contiguous) are dead outside a fix: >= 576 B per site
    const size_t stage = (size_t)((char *)sl.part - (char *)sl.u64r);
    const uint32_t per = (uint32_t)std::max<size_t>(1, stage / per_slice);
    for (uint32_t t0 = 0; t0 < (uint32_t)l.nt; t0 += per) {
        uint32_t n = std::min<uint32_t>(per, l.nt - t0);
        launch_store_gt(sl.g, l, t0, n, elem_bytes, byteswap, sl.u64r, st);
        GFC_CHECK(cudaMemcpyAsync((char *)host + (size_t)t0 * per_slice, sl.u64r, n * per_slice,
                                  cudaMemcpyDeviceToHost, st));
    }
    GFC_CHECK(cudaStreamSynchronize(st));
    return GFC_OK;
}

// Map `bytes` of device memory into the slot pool ahead of time (allocated and
// freed once; the pool keeps it), so admissions do not wait for the mapping.
int batch_warm_pool(gfc_batch *b, size_t bytes) {
    GFC_CHECK(cudaSetDevice(b->dev));
    void *m = nullptr;
    if (cudaMallocFromPoolAsync(&m, bytes, b->pool, b->s) != cudaSuccess) {
        cudaGetLastError();
        set_error("cannot map %zu bytes of device memory for the slot pool", bytes);
        return GFC_ERR_NOMEM;
    }
    GFC_CHECK(cudaFreeAsync(m, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    return GFC_OK;
}
}  // namespace gfc

extern "C" int gfc_batch_download_gt(gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap) {
    if (!b) return GFC_ERR_ARG;
    return batch_download_gt_on(b, slot, host, elem_bytes, byteswap, b->s);
}

extern "C" int gfc_batch_download_links(gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    if (b->activated[slot]) {
        set_error("slot %d is still being fixed (finalize it first)", slot);
        return GFC_ERR_STATE;
    }
    if (!host || (elem_bytes != 8 && elem_bytes != 4)) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    const BSlot &sl = b->hs[slot];
    const Lat &l = sl.l;
    const size_t per_slice = (size_t)l.vs * 4 * 18 * elem_bytes;
    // the working copies (u64r .. g32, contiguous) are dead outside a fix: >= 576 B per site
    const size_t stage = (size_t)((char *)sl.part - (char *)sl.u64r);
    const uint32_t per = (uint32_t)std::max<size_t>(1, stage / per_slice);
    for (uint32_t t0 = 0; t0 < (uint32_t)l.nt; t0 += per) {
        uint32_t n = std::min<uint32_t>(per, l.nt - t0);
        launch_store_links(sl.u, sl.ut, l, t0, n, elem_bytes, byteswap, sl.u64r, b->s);
        GFC_CHECK(cudaMemcpyAsync((char *)host + (size_t)t0 * per_slice, sl.u64r, n * per_slice,
                                  cudaMemcpyDeviceToHost, b->s));
    }
    GFC_CHECK(cudaStreamSynchronize(b->s));
    return GFC_OK;
}

// half-sweeps each timeslice of the slot has received (nt values)
extern "C" int gfc_batch_slice_sweeps(gfc_batch *b, int slot, int *out) {
    int rc = check_slot(b, slot);
    if (rc) return rc;
    if (!out) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    GFC_CHECK(cudaMemcpyAsync(out, b->sweeps + (size_t)slot * b->max_nt, sizeof(int) * b->nt[slot],
                              cudaMemcpyDeviceToHost, b->s));
    GFC_CHECK(cudaStreamSynchronize(b->s));
    return GFC_OK;
}

extern "C" int gfc_batch_status(gfc_batch *b, unsigned *status) {
    if (!b || !status) return GFC_ERR_ARG;
    GFC_CHECK(cudaSetDevice(b->dev));
    GFC_CHECK(cudaMemcpy(status, b->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    GFC_CHECK(cudaMemset(b->status, 0, sizeof(unsigned)));
    return GFC_OK;
}

extern "C" long long gfc_batch_kernel_launches(const gfc_batch *b) { return b ? b->launches : -1; }
extern "C" void *gfc_batch_stream(gfc_batch *b) { return b ? (void *)b->s : nullptr; }

// launch shape (minimum resident CTAs per SM) of the two sweep kernels and the
// half-sweeps per captured round
static bool valid_minb(int m) { return (m >= 1 && m <= 4) || m == 8 || m == 11 || m == 12; }

extern "C" int gfc_batch_set_shape(gfc_batch *b, int minb32, int minb64, int round_sweeps) {
    if (!b || !valid_minb(minb32) || !valid_minb(minb64) || round_sweeps < 1 || round_sweeps > 64)
        return GFC_ERR_ARG;
    b->minb32 = minb32;
    b->minb64 = minb64;
    b->round_k = round_sweeps;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return GFC_OK;
}

// FP64 links staged in shared memory by the batch sweep (1) or not (0)
extern "C" int gfc_batch_set_staging(gfc_batch *b, int stage64) {
    if (!b) return GFC_ERR_ARG;
    b->stage64 = stage64 != 0;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return GFC_OK;
}

extern "C" int gfc_batch_get_shape(const gfc_batch *b, int *minb32, int *minb64, int *stage64, int *round_sweeps) {
    if (!b) return GFC_ERR_ARG;
    if (minb32) *minb32 = b->minb32;
    if (minb64) *minb64 = b->stage64 && b->minb64 <= 4 ? std::min(b->minb64, 3) : b->minb64;
    if (stage64) *stage64 = b->minb64 > 4 ? 1 : b->stage64;
    if (round_sweeps) *round_sweeps = b->round_k;
    return GFC_OK;
}

// Times the batch's launch shapes on a scratch lattice of the given size (seeded
// synthetic links) and keeps the fastest: resident CTAs per SM of the FP32 sweep,
// resident CTAs and shared-memory staging of the FP64 sweep, then half-sweeps per
// captured round.  The batch must have no activated slot; the scratch slot is
// removed again.  times (may be NULL, GFC_BATCH_TUNE_SLOTS entries) receives seconds
// per half-sweep: [0..2] FP32 minb 2,3,4; [3..7] FP64 (minb, staged) (2,0) (3,0)
// (4,0) (2,1) (3,1); [8..10] rounds of 4, 8, 16 half-sweeps; [11..13] FP32 and
// [14..16] FP64 one-warp CTAs, 8, 11, 12 per SM.
extern "C" int gfc_batch_autotune(gfc_batch *b, int ns, int nt, double *times) {
    if (!b) return GFC_ERR_ARG;
    for (int k = 0; k < b->max_slots; k++)
        if (b->used[k] && b->activated[k]) {
            set_error("autotune needs a batch without activated slots");
            return GFC_ERR_STATE;
        }
    double t[GFC_BATCH_TUNE_SLOTS] = {0};
    int slot = -1;
    int rc = gfc_batch_add(b, ns, nt, &slot);
    if (rc) return rc;
    gfc_params pt;
    gfc_params_default(&pt);
    pt.tolerance = 1e-300;   // nothing retires while timing
    gfc_options ot;
    gfc_options_default(&ot);
    ot.switch_e2 = 1e-300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int save32 = b->minb32, save64 = b->minb64, saves = b->stage64, savek = b->round_k;
    auto time_rounds = [&](int prec, double &out) -> int {
        ot.precision = prec;
        int active = 0, r = gfc_batch_round(b, &pt, &ot, &active);   // warm: capture + first round
        if (r) return r;
        GFC_CHECK(cudaEventRecord(e0, b->s));
        for (int q = 0; q < 3; q++)
            if ((r = gfc_batch_round(b, &pt, &ot, &active))) return r;
        GFC_CHECK(cudaEventRecord(e1, b->s));
        GFC_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        GFC_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        out = ms * 1e-3 / (3.0 * b->round_k);
        return GFC_OK;
    };
    int best32 = save32, best64 = save64, bests = saves, bestk = savek;
    auto ce = [](cudaError_t e) { return e == cudaSuccess ? GFC_OK : cuda_fail(e, "cudaEventCreate"); };
    do {
        if ((rc = ce(cudaEventCreate(&e0)))) break;
        if ((rc = ce(cudaEventCreate(&e1)))) break;
        if ((rc = gfc_batch_synth(b, slot, 1, 0.5))) break;
        // FP32 sweep
        if ((rc = gfc_batch_activate(b, slot, GFC_PREC_MIXED))) break;
        double best = 1e30;
        // one-warp shapes first: they share one launch with the FP64 items
        // (k_bsweep_wf, whose shape is the FP64 one, so they are timed in that shape),
        // which saves a launch and a tail per half-sweep when both precisions are
        // active, something a lattice in FP32 alone does not show; a 128-thread shape
        // is kept only if it is more than 2 % faster.  The most resident CTAs come
        // first and a later one-warp shape must be 1 % faster to replace them: on a
        // mix of many lattices 12 per SM measured 2 % faster than 11 or 8, which one
        // lattice alone times within noise of each other.
        const int m32[6] = {12, 11, 8, 2, 3, 4}, i32[6] = {13, 12, 11, 0, 1, 2};
        for (int q = 0; q < 6 && !rc; q++) {
            gfc_batch_set_shape(b, m32[q], m32[q] > 4 ? m32[q] : (save64 > 4 ? 3 : save64), 4);
            rc = time_rounds(GFC_PREC_MIXED, t[i32[q]]);
            const double margin = m32[q] > 4 ? 0.99 : 0.98;
            if (!rc && t[i32[q]] < best * margin) best = t[i32[q]], best32 = m32[q];
        }
        if (rc) break;
        // FP64 sweep
        if ((rc = gfc_batch_activate(b, slot, GFC_PREC_FP64_FAST))) break;
        best = 1e30;
        // one-warp shapes first, most resident first, as for FP32
        const int m64[8] = {12, 11, 8, 2, 3, 4, 2, 3}, st64[8] = {1, 1, 1, 0, 0, 0, 1, 1};
        const int i64[8] = {16, 15, 14, 3, 4, 5, 6, 7};
        for (int q = 0; q < 8 && !rc; q++) {
            gfc_batch_set_shape(b, best32, m64[q], 4);
            gfc_batch_set_staging(b, st64[q]);
            rc = time_rounds(GFC_PREC_FP64_FAST, t[i64[q]]);
            if (!rc && t[i64[q]] < best * 0.99) best = t[i64[q]], best64 = m64[q], bests = st64[q];
        }
        if (rc) break;
        // half-sweeps per round (FP64 work; the per-round compaction is amortised)
        best = 1e30;
        const int ks[3] = {4, 8, 16};
        gfc_batch_set_staging(b, bests);
        for (int q = 0; q < 3 && !rc; q++) {
            gfc_batch_set_shape(b, best32, best64, ks[q]);
            rc = time_rounds(GFC_PREC_FP64_FAST, t[8 + q]);
            if (!rc && t[8 + q] < best * 0.98) best = t[8 + q], bestk = ks[q];
        }
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    k_set_state<<<(nt + 127) / 128, 128, 0, b->s>>>(b->state, slot * b->max_nt, nt, SS_EMPTY);
    b->activated[slot] = 0;
    int rc2 = gfc_batch_remove(b, slot);
    if (!rc) rc = rc2;
    if (rc) {
        gfc_batch_set_shape(b, save32, save64, savek);
        gfc_batch_set_staging(b, saves);
        return rc;
    }
    gfc_batch_set_shape(b, best32, best64, bestk);
    gfc_batch_set_staging(b, bests);
    if (times)
        for (int q = 0; q < GFC_BATCH_TUNE_SLOTS; q++) times[q] = t[q];
    return GFC_OK;
}

// Run every activated slot to retirement (or max_sweeps) and finalise it.
// reports[slot] is filled for every slot that was active; returns the number of
// rounds, or an error.
extern "C" int gfc_batch_fix_all(gfc_batch *b, const gfc_params *p, const gfc_options *o, gfc_report *reports) {
    if (!b || !p) return GFC_ERR_ARG;
    if (!gfc_params_valid(p)) return GFC_FIX_BAD_PARAMS;
    std::vector<int> act(b->max_slots, 0);
    for (int s = 0; s < b->max_slots; s++) act[s] = b->used[s] && b->activated[s];
    const int max_rounds = (int)(p->max_sweeps_to_fix / (unsigned)b->round_k) + 1;
    int rounds = 0, active = 1;
    while (active > 0 && rounds < max_rounds) {
        int rc = gfc_batch_round(b, p, o, &active);
        if (rc) return rc;
        rounds++;
    }
    for (int s = 0; s < b->max_slots; s++)
        if (act[s]) {
            int done = 0;
            gfc_batch_slot_done(b, s, &done);
            int rc = gfc_batch_finalize(b, s, reports ? reports + s : nullptr);
            if (rc) return rc;
            if (reports && !done) reports[s].status = GFC_FIX_NOT_CONVERGED;
        }
    return rounds;
}
