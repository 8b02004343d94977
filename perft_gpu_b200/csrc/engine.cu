// B200 perft engine: level-synchronous tree expansion with a fused,
// count-only last ply.
//
// What it replaces in the reference (ankan-ban/perft_gpu):
//   perft_bb_gpu_simple / _hash BFS drivers (perft_bb.h:1027-1138,
//   1242-1589), the per-level kernels makemove_and_count_moves_single_level
//   (perft_bb.h:601-625), generate_moves_single_level (perft_bb.h:983-996),
//   the leaf pass makeMove_and_perft_single_level_indices (perft_bb.h:412-446)
//   and moderngpu's ScanD + IntervalExpandDGenValues (perft_bb.h:1088-1124).
//
// Design (B200-first):
//   * Boards are side-relative (movegen.cuh), so no kernel branches on the
//     side to move.
//   * A level is a structure-of-arrays buffer in HBM: the boards as three
//     arrays of 16-byte plane pairs (128-bit loads and stores), plus the move
//     count and root id of each node.  Every node of a level has
//     the same remaining depth (roots are grouped by depth).
//   * One exclusive scan of the move counts turns a level into a flat list
//     of (parent, move) items.  Items are cut into fixed tiles of TILE_CAP;
//     the scan also records the first parent of every tile, so the tile
//     kernel needs no search and no parent-index expansion buffer.
//   * The tile kernel is persistent (one wave of CTAs sized by occupancy)
//     and steals tiles from an atomic counter.  Per tile it stages the
//     parents in shared memory, generates their moves into a compact shared
//     item list (only the moves inside the tile window), then every thread
//     takes items: make the move, count the child's legal moves.  Interior
//     plies write the child (coalesced: item order is child order) and its
//     count; the last ply only sums counts per root, warp-aggregated with
//     match/reduce before a shared-memory accumulator and one global atomic
//     per root run.
//   * When a level does not fit the HBM arena, its item range is split at
//     tile boundaries and the chunks are expanded depth-first.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/perft_b200.h"
#include "movegen.cuh"

namespace pg {
void build_tables();
}  // namespace pg

using namespace pg;

namespace {

// ------------------------------------------------------------- constants
#ifndef PG_TILE_CAP_LOG2
#define PG_TILE_CAP_LOG2 13
#endif
#ifndef PG_TILE_MINB
#define PG_TILE_MINB 3
#endif
#ifndef PG_ONE_RUN_VOTE
#define PG_ONE_RUN_VOTE 1  // one block vote for windows whose parents share one root
#endif
#ifndef PG_ONE_RUN_SUM
#define PG_ONE_RUN_SUM 1  // such windows sum their counts with a plain warp reduction
#endif
#ifndef PG_MIRRORED_STAGE
#define PG_MIRRORED_STAGE 1  // parents staged mirrored: children are made in their own frame
#endif
#ifndef PG_KNOWN_KINGS
#define PG_KNOWN_KINGS 1  // (with mirrored staging) the count gets both king squares from the parent
#endif
#ifndef PG_KNOWN_OCC
#define PG_KNOWN_OCC 1  // (with known kings) and the occupancy and opponent set from make-move
#endif
#ifndef PG_TILE_NT
#define PG_TILE_NT 256
#endif
constexpr int TILE_NT = PG_TILE_NT;  // threads per tile CTA
constexpr int TILE_CAP_LOG2 = PG_TILE_CAP_LOG2;  // largest tile: 2^TILE_CAP_LOG2 items
constexpr int TILE_CAP = 1 << TILE_CAP_LOG2;
constexpr int TILE_MIN_LOG2 = 10;  // small levels use tiles down to 1024 items to fill every SM
constexpr u64 MAX_TILES_PER_NODE_DIV = 1ull << TILE_MIN_LOG2;
constexpr int TILE_MAXP = TILE_NT;
constexpr int TILE_MINB = PG_TILE_MINB;          // resident CTAs per SM the register budget targets
constexpr int MAX_LEGAL_MOVES = 218;

constexpr int SCAN_NT = 512;
constexpr int SCAN_IPT = 16;
constexpr int SCAN_CHUNK = SCAN_NT * SCAN_IPT;
constexpr int SCAN_TOP_NT = 1024;

constexpr u32 DERR_GEN_MISMATCH = 1u;
constexpr u32 DERR_BAD_ITEM = 2u;
constexpr u32 DERR_BAD_POSITION = 4u;

enum { MODE_EXPAND = 0, MODE_LEAF = 1 };

// Bytes of one level node: 6 planes + count + root + scan entry, plus its
// share of the tile index (4 B per TILE_CAP items, up to 218 items a node)
// and of the scan's block sums, rounded up.
constexpr u64 NODE_BYTES = 6 * 8 + 4 + 4 + 8 + 1;  // (tile index sized for the smallest tile: < 1 B/node)

// ------------------------------------------------------- level node boards
// A level's boards in HBM are a structure of arrays of plane pairs: pair j of
// node g (planes 2j and 2j+1: mine/pawns, knights/bq, rq/kings) is one
// 16-byte vector at pp[j * stride + g].  A node is written with three 128-bit
// stores and read with three 128-bit loads, and a warp's 32 consecutive nodes
// touch 512 contiguous bytes per pair.  48 bytes per node, as six u64 planes.
__device__ __forceinline__ void level_put(u64 *planes, u64 stride, u64 g, const Board &b)
{
    ulonglong2 *pp = reinterpret_cast<ulonglong2 *>(planes);
    pp[g] = make_ulonglong2(b.mine, b.pawns);
    pp[stride + g] = make_ulonglong2(b.knights, b.bq);
    pp[2 * stride + g] = make_ulonglong2(b.rq, b.kings);
}

__device__ __forceinline__ Board level_get(const u64 *planes, u64 stride, u64 g)
{
    const ulonglong2 *pp = reinterpret_cast<const ulonglong2 *>(planes);
    const ulonglong2 a = pp[g], c = pp[stride + g], d = pp[2 * stride + g];
    return Board{a.x, a.y, c.x, c.y, d.x, d.y};
}

// --------------------------------------------------------- block helpers
template <int NT>
__device__ __forceinline__ u64 block_excl_scan_u64(u64 v, u64 *sw, u64 &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u64 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u64 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sw[w] = x;
    __syncthreads();
    if (w == 0) {
        u64 t = lane < NT / 32 ? sw[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u64 y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NT / 32) sw[lane] = t;
    }
    __syncthreads();
    const u64 warpOff = w ? sw[w - 1] : 0;
    total = sw[NT / 32 - 1];
    __syncthreads();
    return warpOff + x - v;
}

// Exclusive count of set flags over the block; total returned in *total.
template <int NT>
__device__ __forceinline__ int block_excl_count(bool flag, int *sw, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned b = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) sw[w] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) {
        off += (i < w) ? sw[i] : 0;
        tot += sw[i];
    }
    __syncthreads();
    total = tot;
    return off + __popc(b & ((1u << lane) - 1u));
}

// ------------------------------------------------------------------ scan
// Exclusive scan of u32 move counts into u64 item offsets (n + 1 entries,
// the last one the total), plus the first parent of every TILE_CAP tile.
__global__ void __launch_bounds__(SCAN_NT) k_scan_reduce(const u32 *__restrict__ cnt, u64 n,
                                                         u64 *__restrict__ bsum)
{
    __shared__ u64 sw[SCAN_NT / 32];
    const u64 base = (u64)blockIdx.x * SCAN_CHUNK;
    u64 s = 0;
    for (int i = threadIdx.x; i < SCAN_CHUNK; i += SCAN_NT) {
        const u64 k = base + i;
        if (k < n) s += cnt[k];
    }
    u64 total;
    block_excl_scan_u64<SCAN_NT>(s, sw, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_TOP_NT) k_scan_top(u64 *__restrict__ bsum, u64 nb,
                                                          u64 *__restrict__ totalOut)
{
    __shared__ u64 sw[SCAN_TOP_NT / 32];
    const u64 per = (nb + SCAN_TOP_NT - 1) / SCAN_TOP_NT;
    const u64 b0 = per * threadIdx.x, b1 = min(b0 + per, nb);
    u64 s = 0;
    for (u64 i = b0; i < b1; i++) s += bsum[i];
    u64 total;
    u64 run = block_excl_scan_u64<SCAN_TOP_NT>(s, sw, total);
    for (u64 i = b0; i < b1; i++) {
        const u64 v = bsum[i];
        bsum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) *totalOut = total;
}

__global__ void __launch_bounds__(SCAN_NT) k_scan_apply(const u32 *__restrict__ cnt, u64 n,
                                                        const u64 *__restrict__ bsum,
                                                        u64 *__restrict__ scan,
                                                        u32 *__restrict__ tileFirst, int capLog2)
{
    __shared__ u32 s[SCAN_CHUNK];
    __shared__ u64 sw[SCAN_NT / 32];
    const u64 base = (u64)blockIdx.x * SCAN_CHUNK;
    for (int i = threadIdx.x; i < SCAN_CHUNK; i += SCAN_NT) {
        const u64 k = base + i;
        s[i] = k < n ? cnt[k] : 0u;
    }
    __syncthreads();
    u64 local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IPT; k++) local += s[threadIdx.x * SCAN_IPT + k];
    u64 total;
    u64 run = bsum[blockIdx.x] + block_excl_scan_u64<SCAN_NT>(local, sw, total);
    for (int k = 0; k < SCAN_IPT; k++) {
        const u64 idx = base + (u64)threadIdx.x * SCAN_IPT + k;
        if (idx >= n) break;
        const u32 c = s[threadIdx.x * SCAN_IPT + k];
        scan[idx] = run;
        if (c) {
            const u64 t0 = (run + (1ull << capLog2) - 1) >> capLog2;
            const u64 t1 = (run + c - 1) >> capLog2;
            for (u64 t = t0; t <= t1; t++) tileFirst[t] = (u32)idx;
        }
        run += c;
    }
}

// ----------------------------------------------------------------- roots
__global__ void k_init_roots(const u64 *__restrict__ pos48, const u32 *__restrict__ ids, u32 n,
                             u64 *__restrict__ planes, u64 stride, u32 *__restrict__ cnt,
                             u32 *__restrict__ root, int depth,
                             unsigned long long *__restrict__ rootCounts, u32 *err)
{
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 id = ids[i];
    u64 p[6];
#pragma unroll
    for (int k = 0; k < 6; k++) p[k] = pos48[6 * (u64)id + k];
    u32 c = 0;
    Board b = from_pos48(p);
    if (validate_pos48(p) != 0) {
        atomicOr(err, DERR_BAD_POSITION);
    } else {
        c = count_moves<SV_KOGGE>(b);
    }
    level_put(planes, stride, i, b);
    cnt[i] = c;
    root[i] = id;
    if (depth == 0) rootCounts[id] = 1ull;
    if (depth == 1) rootCounts[id] = c;
}

// ------------------------------------------- device-driven level pipeline
// The scan of level k runs with a fixed grid (grid-stride over chunks), its
// top block computes the total and bump-allocates level k+1 and that
// level's scan buffers from a device-resident plan.  No host round trip
// separates the plies, so a whole perft is one captured CUDA graph.  If the
// region is exhausted the plan's overflow flag is raised, every following
// level is empty, and the host reruns the batch on the host-driven path.
// A level whose sizes and buffers are decided on the device (device-driven
// pipeline, no host round trip between plies).
struct LevelDesc {
    u64 *planes;
    u64 stride;
    u32 *cnt;
    u32 *root;
    u64 n;        // nodes: the previous ply's children, then the roots joining here
    u64 nChild;   // children written by the previous ply's tile kernel
    u64 *pscan;
    u32 *tileFirst;
    u64 *bsum;
    u64 total;
    int capLog2;  // tile size of this level's items
};

struct TileParams {
    const u64 *ppl;   // parent planes, plane i at ppl + i * pstride
    u64 pstride;
    const u64 *pscan; // nParents + 1 item offsets
    const u32 *proot;  // root id of each parent; null: sums go to the parent's own slot
    u64 nParents;
    const u32 *tileFirst;  // indexed by absolute tile number
    u64 itemBase;     // first item of this launch (multiple of the tile size)
    u64 itemEnd;      // one past the last item
    int capLog2;      // tile size of this level (the scan's tileFirst granularity)
    u32 *tileCounter; // work-stealing cursor, zeroed before launch
    // interior ply outputs (child index = item - itemBase)
    u64 *cpl;
    u64 cstride;
    u32 *ccnt;
    u32 *croot;
    // last ply output
    unsigned long long *rootCounts;
    u32 *err;
    // serving: pending-node counter of each query slot (TRACK kernels only)
    unsigned long long *pending;
    // device-driven DD_SHARED launches: the plan's entry for this launch
    const struct TileParams *planEntry;
};


constexpr int DD_MAX_LEVELS = 24;
// Largest predicted tree (bytes of materialised plies) run as a graph, on top
// of the arena check: no limit unless PERFT_DD_MAX_GB sets one.
constexpr double DD_MAX_BYTES_DEFAULT = 1e30;
// Plies predicted to have fewer items than this read their launch
// parameters through shared memory instead of a constant-bank copy node.
constexpr double DD_CONST_MIN_ITEMS = double(1u << 22);
struct DevPlan {
    char *base;
    u64 cap;
    u64 bump;
    u32 overflow;
    u32 tileTarget;  // smallest tile count a level should have (2 x resident CTAs)
    LevelDesc lv[DD_MAX_LEVELS];
    // roots that join level k (their depth is the level's remaining depth)
    u32 joinN[DD_MAX_LEVELS];
    const u32 *joinIds[DD_MAX_LEVELS];
    int capMax[DD_MAX_LEVELS];  // largest tile (log2 items) for the items of level k
    // the tile launch of level k's items, completed on the device by the scan
    // (level pointers and sizes) and copied into c_ddTile before that launch
    TileParams tp[DD_MAX_LEVELS];
    u32 *tileCounter;  // the tile launches' work-stealing cursor, reset by each scan
};

// The parameters of the device-driven tile launch about to run.  A graph
// copies the plan's entry for the level here (a device-to-device copy node)
// before each tile launch, so the kernel reads them from the constant bank,
// as a plain launch reads its parameters, instead of holding plan pointers
// in registers or shared memory.  Only the device-driven graphs use it, and
// they run one at a time on the engine's stream.
__constant__ TileParams c_ddTile;

__device__ __forceinline__ void *dd_take(DevPlan *plan, u64 bytes)
{
    const u64 a = (plan->bump + 255) & ~255ULL;
    if (a + bytes > plan->cap) {
        plan->overflow = 1;
        return nullptr;
    }
    plan->bump = a + bytes;
    return plan->base + a;
}

__global__ void __launch_bounds__(SCAN_NT) k_dd_scan_reduce(DevPlan *plan, int lv)
{
    __shared__ u64 sw[SCAN_NT / 32];
    const LevelDesc &L = plan->lv[lv];
    const u64 n = L.n, nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    for (u64 b = blockIdx.x; b < nb; b += gridDim.x) {
        const u64 base = b * SCAN_CHUNK;
        u64 s = 0;
        for (int i = threadIdx.x; i < SCAN_CHUNK; i += SCAN_NT) {
            const u64 k = base + i;
            if (k < n) s += L.cnt[k];
        }
        u64 total;
        block_excl_scan_u64<SCAN_NT>(s, sw, total);
        if (threadIdx.x == 0) L.bsum[b] = total;
    }
}

__device__ void dd_plan_level(DevPlan *plan, int lv, int last, u64 total);

__global__ void __launch_bounds__(SCAN_TOP_NT) k_dd_scan_top(DevPlan *plan, int lv, int last)
{
    __shared__ u64 sw[SCAN_TOP_NT / 32];
    LevelDesc &L = plan->lv[lv];
    const u64 n = L.n, nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    const u64 per = (nb + SCAN_TOP_NT - 1) / SCAN_TOP_NT;
    const u64 b0 = per * threadIdx.x, b1 = min(b0 + per, nb);
    u64 s = 0;
    for (u64 i = b0; i < b1; i++) s += L.bsum[i];
    u64 total;
    u64 run = block_excl_scan_u64<SCAN_TOP_NT>(s, sw, total);
    for (u64 i = b0; i < b1; i++) {
        const u64 v = L.bsum[i];
        L.bsum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) dd_plan_level(plan, lv, last, total);
}

// Whole-level scan in one block: the total, the tile size and the next level
// (dd_plan_level), then the offsets and tile index, 1024 nodes per pass.
// Used for levels predicted small, where three launches (each with its own
// latency) would cost more than the work; correct for any size.
__global__ void __launch_bounds__(1024) k_dd_scan_small(DevPlan *plan, int lv, int last)
{
    __shared__ u64 sw[32];
    __shared__ int sCap;
    LevelDesc &L = plan->lv[lv];
    const u64 n = L.n;
    u64 s = 0;
    for (u64 i = threadIdx.x; i < n; i += 1024) s += L.cnt[i];
    u64 total;
    block_excl_scan_u64<1024>(s, sw, total);
    if (threadIdx.x == 0) {
        dd_plan_level(plan, lv, last, total);
        sCap = L.capLog2;
    }
    __syncthreads();
    const int cl = sCap;
    u64 base = 0;
    for (u64 c0 = 0; c0 < n; c0 += 1024) {
        const u64 i = c0 + threadIdx.x;
        const u32 c = i < n ? L.cnt[i] : 0u;
        u64 tot;
        const u64 run = base + block_excl_scan_u64<1024>(c, sw, tot);
        if (i < n) {
            L.pscan[i] = run;
            if (c) {
                const u64 t0 = (run + (1ull << cl) - 1) >> cl;
                const u64 t1 = (run + c - 1) >> cl;
                for (u64 t = t0; t <= t1; t++) L.tileFirst[t] = (u32)i;
            }
        }
        base += tot;
    }
}

// Top-of-scan bookkeeping of a device-driven level (one thread): the level's
// total and tile size, then the next level's buffers from the plan's bump
// allocator (children plus the roots joining there).
__device__ void dd_plan_level(DevPlan *plan, int lv, int last, u64 total)
{
    LevelDesc &L = plan->lv[lv];
    const u64 n = L.n;
    if (n) L.pscan[n] = total;
    L.total = plan->overflow ? 0 : total;
    int cap = plan->capMax[lv] ? plan->capMax[lv] : TILE_CAP_LOG2;
    while (cap > TILE_MIN_LOG2 && (total >> cap) < plan->tileTarget) cap--;
    L.capLog2 = cap;
    *plan->tileCounter = 0;  // the next launch is this level's tile launch
    TileParams &T = plan->tp[lv];  // host fields (cursor, outputs, error word) come from the template
    T.ppl = L.planes;
    T.pstride = L.stride;
    T.pscan = L.pscan;
    T.proot = L.root;
    T.nParents = L.n;
    T.tileFirst = L.tileFirst;
    T.itemBase = 0;
    T.itemEnd = L.total;
    T.capLog2 = cap;
    if (last) return;
    LevelDesc &C = plan->lv[lv + 1];
    const u64 m = L.total + plan->joinN[lv + 1];
    C.n = m;
    C.nChild = L.total;
    C.stride = (m + 31) & ~31ULL;
    C.total = 0;
    C.planes = (u64 *)dd_take(plan, 48 * C.stride);
    C.cnt = (u32 *)dd_take(plan, 4 * C.stride);
    C.root = (u32 *)dd_take(plan, 4 * C.stride);
    C.pscan = (u64 *)dd_take(plan, 8 * (m + 1));
    C.tileFirst = (u32 *)dd_take(plan, 4 * ((m * MAX_LEGAL_MOVES) / MAX_TILES_PER_NODE_DIV + 2));
    C.bsum = (u64 *)dd_take(plan, 8 * ((m + SCAN_CHUNK - 1) / SCAN_CHUNK + 1));
    if (plan->overflow) {
        C.n = 0;
        L.total = 0;  // nothing is expanded into a level that does not exist
    }
    T.itemEnd = L.total;
    T.cpl = C.planes;
    T.cstride = C.stride;
    T.ccnt = C.cnt;
    T.croot = C.root;
}

__global__ void __launch_bounds__(SCAN_NT) k_dd_scan_apply(DevPlan *plan, int lv)
{
    __shared__ u32 s[SCAN_CHUNK];
    __shared__ u64 sw[SCAN_NT / 32];
    const LevelDesc &L = plan->lv[lv];
    const u64 n = L.n, nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    for (u64 b = blockIdx.x; b < nb; b += gridDim.x) {
        const u64 base = b * SCAN_CHUNK;
        for (int i = threadIdx.x; i < SCAN_CHUNK; i += SCAN_NT) {
            const u64 k = base + i;
            s[i] = k < n ? L.cnt[k] : 0u;
        }
        __syncthreads();
        u64 local = 0;
#pragma unroll
        for (int k = 0; k < SCAN_IPT; k++) local += s[threadIdx.x * SCAN_IPT + k];
        u64 total;
        u64 run = L.bsum[b] + block_excl_scan_u64<SCAN_NT>(local, sw, total);
        for (int k = 0; k < SCAN_IPT; k++) {
            const u64 idx = base + (u64)threadIdx.x * SCAN_IPT + k;
            if (idx >= n) break;
            const u32 c = s[threadIdx.x * SCAN_IPT + k];
            L.pscan[idx] = run;
            if (c) {
                const int cl = L.capLog2;
                const u64 t0 = (run + (1ull << cl) - 1) >> cl;
                const u64 t1 = (run + c - 1) >> cl;
                for (u64 t = t0; t <= t1; t++) L.tileFirst[t] = (u32)idx;
            }
            run += c;
        }
        __syncthreads();
    }
}

// Roots joining level lv of a device-driven run: written behind the
// children, from the position array (as k_init_roots does).  Nothing is
// written into a level that overflowed the plan.
__global__ void k_dd_join(DevPlan *plan, int lv, const u64 *__restrict__ pos48, u32 *err)
{
    const LevelDesc &C = plan->lv[lv];
    const u32 nj = plan->joinN[lv];
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nj || C.n == 0 || plan->overflow) return;
    const u32 id = plan->joinIds[lv][i];
    u64 p[6];
#pragma unroll
    for (int k = 0; k < 6; k++) p[k] = pos48[6 * (u64)id + k];
    u32 c = 0;
    const Board b = from_pos48(p);
    if (validate_pos48(p) != 0) atomicOr(err, DERR_BAD_POSITION);
    else c = count_moves<SV_KOGGE>(b);
    const u64 g = C.nChild + i;
    level_put(C.planes, C.stride, g, b);
    C.cnt[g] = c;
    C.root[g] = id;
}

// ------------------------------------------------------------ tile kernel



// Emits a parent's moves, keeping only those whose global item index falls
// inside [lo, hi): the window of the current tile.
// Positions are relative to the window start: a parent starts at most
// MAX_LEGAL_MOVES items before it and a window holds at most TILE_CAP items,
// so 32 bits hold them and one unsigned compare does the bounds test.
struct WindowSink {
    u32 *items;
    int rel;  // next move's position relative to the window start
    u32 n;    // window length
    u32 tag;
    __device__ __forceinline__ void operator()(u32 m)
    {
        if ((u32)rel < n) items[rel] = tag | m;
        ++rel;
    }
};

// TRACK (serving): besides the counts, every root run also accumulates the
// change of its query's pending-node counter: +1 per child written, -1 when
// a parent's last item is processed.  The counter reaching zero means the
// query's subtree is fully counted.
// DD: 0 for plain launches (parameters in the parameter bank); DD_SHARED or
// DD_CONST for the device-driven graph's launches (below).
enum { DD_NONE = 0, DD_SHARED = 1, DD_CONST = 2 };
template <int MODE, int SV, bool TRACK = false, int DD = DD_NONE>
__global__ void __launch_bounds__(TILE_NT, TILE_MINB) k_tile(const TileParams Pin)
{
    // Device-driven launches take the level pointers and sizes from the plan:
    //  * DD_CONST reads them from the constant bank (c_ddTile, which the graph
    //    fills by a copy node before the launch), exactly as a plain launch
    //    reads its parameter bank.  Used for large plies: held in registers
    //    across the make-and-count loop the pointers compete with the count at
    //    the 80-register cap (5% slower), and read from shared memory they
    //    still cost 1.3%; from the constant bank the count-only launch of the
    //    4096-position batch takes the same time as a plain launch.
    //  * DD_SHARED reads the plan entry into shared memory at the start of the
    //    launch.  Used for small plies, where the copy node's few microseconds
    //    would cost more than they save.
    __shared__ TileParams sP;
    if (DD == DD_SHARED) {
        if (threadIdx.x == 0) sP = *Pin.planEntry;
        __syncthreads();
    }
    const TileParams &P = DD == DD_CONST ? c_ddTile : (DD == DD_SHARED ? sP : Pin);
    __shared__ u64 sb[6][TILE_MAXP];
    // king squares in the children's frame: the side to move there (the
    // parent's opponent) and the parent's mover
    __shared__ uint8_t skO[PG_KNOWN_KINGS ? TILE_MAXP : 1], skS[PG_KNOWN_KINGS ? TILE_MAXP : 1];
    __shared__ u64 sqEnd[TRACK ? TILE_MAXP : 1];
    __shared__ int sdelta[TRACK ? TILE_MAXP : 1];
    __shared__ u32 sroot[TILE_MAXP];
    __shared__ u32 srun[TILE_MAXP];
    __shared__ u32 srunRoot[TILE_MAXP];
    __shared__ unsigned long long sacc[TILE_MAXP];
    extern __shared__ __align__(16) u32 sitems[];  // TILE_CAP items (dynamic: may exceed 48 KB)
    __shared__ int swarp[TILE_NT / 32];
    __shared__ u32 sTile;

    const int tid = threadIdx.x, lane = tid & 31;
    const int capLog2 = P.capLog2;
    const u64 tile0 = P.itemBase >> capLog2;
    const u64 nTiles = (P.itemEnd - P.itemBase + (1ull << capLog2) - 1) >> capLog2;

    for (;;) {
        if (tid == 0) sTile = atomicAdd(P.tileCounter, 1u);
        __syncthreads();
        const u64 tl = sTile;
        if (tl >= nTiles) break;
        const u64 iBeg = P.itemBase + (tl << capLog2);
        const u64 iEnd = min(iBeg + ((u64)1 << capLog2), P.itemEnd);
        u64 p = P.tileFirst[tile0 + tl];

        for (;;) {
            // ---- stage the parents that own items of this window
            const u64 q = p + tid;
            u64 qBeg = 0, qEnd = 0;
            bool valid = false;
            if (q < P.nParents) {
                qBeg = P.pscan[q];
                valid = qBeg < iEnd;
            }
            const int nP = __syncthreads_count(valid);
            if (valid) {
                qEnd = P.pscan[q + 1];
                if (TRACK) sqEnd[tid] = qEnd;
                // mirrored staging: the per-parent flips here replace six
                // byte swaps per child in make-move
                const Board lb = level_get(P.ppl, P.pstride, q);
                const Board pb = PG_MIRRORED_STAGE ? flip_board(lb) : lb;
                sb[0][tid] = pb.mine;
                sb[1][tid] = pb.pawns;
                sb[2][tid] = pb.knights;
                sb[3][tid] = pb.bq;
                sb[4][tid] = pb.rq;
                sb[5][tid] = pb.kings;
                if (PG_KNOWN_KINGS && PG_MIRRORED_STAGE) {
                    skO[tid] = (uint8_t)ctz(pb.kings & ~pb.mine);
                    skS[tid] = (uint8_t)ctz(pb.kings & pb.mine);
                }
                sroot[tid] = P.proot ? P.proot[q] : (u32)q;  // no root array: account to the parent itself
            }
            const u64 sBeg = max(P.pscan[p], iBeg);
            const u64 sEnd = min(P.pscan[p + nP], iEnd);
            __syncthreads();

            int nRuns = 0;
            if (MODE == MODE_LEAF || TRACK) {
                // parents are ordered by root: number the runs of equal roots.
                // Usually the whole window belongs to one root, which one
                // block vote settles without the two-barrier run count.
                if (PG_ONE_RUN_VOTE && nP > 0 && __syncthreads_and(!valid || sroot[tid] == sroot[0])) {
                    nRuns = 1;
                    if (valid) srun[tid] = 0;
                    if (tid == 0) {
                        srunRoot[0] = sroot[0];
                        sacc[0] = 0ull;
                        if (TRACK) sdelta[0] = 0;
                    }
                } else {
                    const bool head = valid && (tid == 0 || sroot[tid] != sroot[tid - 1]);
                    const int r = block_excl_count<TILE_NT>(head, swarp, nRuns);
                    if (valid) srun[tid] = head ? r : r - 1;
                    if (head) {
                        srunRoot[r] = sroot[tid];
                        sacc[r] = 0ull;
                        if (TRACK) sdelta[r] = 0;
                    }
                }
            }

            // ---- generate the window's moves into the shared item list
            // parents without items (none legal, or answered by the table) generate nothing
            if (valid && qEnd > qBeg && qEnd > sBeg && qBeg < sEnd) {
                const Board sbt{sb[0][tid], sb[1][tid], sb[2][tid], sb[3][tid], sb[4][tid], sb[5][tid]};
                const Board b = PG_MIRRORED_STAGE ? flip_board(sbt) : sbt;
                WindowSink sink{sitems, (int)((long long)qBeg - (long long)sBeg), (u32)(sEnd - sBeg), (u32)tid << 16};
                gen_moves<SV, PG_MOVER_BITS>(b, sink);  // items carry the mover's planes
                if ((long long)sink.rel != (long long)qEnd - (long long)sBeg) atomicOr(P.err, DERR_GEN_MISMATCH);
            }
            __syncthreads();

            // ---- every thread takes items: make, count, write or sum
            const int nItems = (int)(sEnd - sBeg);
            for (int j0 = 0; j0 < nItems; j0 += TILE_NT) {
                const int j = j0 + tid;
                const bool act = j < nItems;
                u32 cnt = 0;
                int pl = 0;
                if (act) {
                    const u32 it = sitems[j];  // move (bits 0-15), parent slot (16-23), mover planes (24-28)
                    pl = (int)((it >> 16) & 0xFFu);
                    if (pl < nP) {
                        const Board b{sb[0][pl], sb[1][pl], sb[2][pl], sb[3][pl], sb[4][pl], sb[5][pl]};
                        Board ch;
                        if (PG_KNOWN_KINGS && PG_MIRRORED_STAGE && PG_KNOWN_OCC) {
                            int tk;
                            u64 occ, theirs;
                            ch = make_child_mirrored(b, it, &tk, skS[pl], &occ, &theirs);
                            cnt = count_moves_ko<SV>(ch, skO[pl], tk, occ, theirs);
                        } else if (PG_KNOWN_KINGS && PG_MIRRORED_STAGE) {
                            int tk;
                            ch = make_child_mirrored(b, it, &tk, skS[pl]);
                            cnt = count_moves_k<SV>(ch, skO[pl], tk);
                        } else {
                            ch = PG_MIRRORED_STAGE ? make_child_mirrored(b, it) : make_child<PG_MOVER_BITS>(b, it);
                            cnt = count_moves<SV>(ch);
                        }
                        if (MODE == MODE_EXPAND) {
                            const u64 g = sBeg + (u64)j - P.itemBase;
                            level_put(P.cpl, P.cstride, g, ch);
                            P.ccnt[g] = cnt;
                            P.croot[g] = sroot[pl];
                        }
                    } else {
                        atomicOr(P.err, DERR_BAD_ITEM);
                        pl = 0;
                    }
                }
                if (PG_ONE_RUN_SUM && MODE == MODE_LEAF && !TRACK && nRuns == 1) {
                    // the whole window belongs to one root: a plain warp sum
                    // (idle lanes hold 0), no grouping by root
                    const u32 sum = __reduce_add_sync(0xffffffffu, cnt);
                    if (lane == 0 && sum) atomicAdd(&sacc[0], (unsigned long long)sum);
                } else if (MODE == MODE_LEAF || TRACK) {
                    const u32 key = act ? srun[pl] : 0xFFFFFFFFu;
                    const unsigned peers = __match_any_sync(0xffffffffu, key);
                    if (MODE == MODE_LEAF) {
                        const u32 sum = __reduce_add_sync(peers, cnt);
                        if (act && lane == __ffs(peers) - 1) atomicAdd(&sacc[key], (unsigned long long)sum);
                    }
                    if (TRACK) {
                        const bool lastOfParent = act && (sBeg + (u64)j + 1 == sqEnd[pl]);
                        const int d = (act && MODE == MODE_EXPAND ? 1 : 0) - (lastOfParent ? 1 : 0);
                        const int dsum = __reduce_add_sync(peers, d);
                        if (act && lane == __ffs(peers) - 1 && dsum) atomicAdd(&sdelta[key], dsum);
                    }
                }
            }
            __syncthreads();
            if (MODE == MODE_LEAF && tid < nRuns) atomicAdd(&P.rootCounts[srunRoot[tid]], sacc[tid]);
            if (TRACK && tid < nRuns && sdelta[tid])
                atomicAdd(&P.pending[srunRoot[tid]], (unsigned long long)(long long)sdelta[tid]);
            if (sEnd >= iEnd || p + nP >= P.nParents) break;
            p += nP;
            __syncthreads();
        }
        __syncthreads();
    }
}

// ============================================================ small trees
// One position of depth 2..5 in one launch, with no level buffers.  The level
// pipeline spends such a tree's time on per-ply latency: a scan and a tile
// launch per ply, each a few microseconds on a handful of busy SMs.  Here
// each CTA takes whole subtrees rooted `depth - r` plies below the position
// (r = 3, or 2 at depth 2) and counts each one in shared memory:
//   1. thread 0 generates the subtree root's moves;
//   2. one thread per move makes the child and counts the child's moves (at
//      r = 2 these counts are the subtree's perft);
//   3. a block scan of those counts places the grandchildren, and one thread
//      per child generates the child's moves into a window of the item list;
//   4. every thread takes items: make the grandchild, count its moves, sum.
// Every CTA lists the subtree roots for itself (the position's moves, and at
// depth 5 its children's moves), so no CTA waits for another; the last CTA
// to finish sums the per-CTA partial counts.  The move generator, make-move
// and count are the level pipeline's own functions.
#ifndef PG_SMALL_NT
#define PG_SMALL_NT 128
#endif
constexpr int SMALL_NT = PG_SMALL_NT;  // threads per CTA: small CTAs put more subtrees in flight
constexpr int SMALL_MINB = 512 / SMALL_NT;
constexpr int SMALL_MAX_DEPTH = 5;
constexpr u32 SMALL_LIST_CAP = 4096;  // subtree roots one CTA can list (depth 5)
constexpr u32 SMALL_WIN = 2048;       // items per window of a subtree's last ply
constexpr size_t SMALL_DYN_SMEM = sizeof(u32) * (SMALL_LIST_CAP + SMALL_WIN);
constexpr int SMALL_MAX_GRID = 1024;
constexpr u32 SMALL_OVERFLOW = 1u << 8;  // more subtree roots than the list holds: not counted

struct SmallState {
    unsigned long long partial[SMALL_MAX_GRID];  // per CTA
    unsigned long long count;                    // the last CTA's sum
    u32 flags;    // 0, SMALL_OVERFLOW or DERR_BAD_POSITION (written by the last CTA)
    u32 done;     // CTAs finished; atomicInc wraps it back to 0 for the next launch
    u32 flagAcc;  // flags raised by any CTA; the last CTA reads and clears it
};

// Exclusive block sum of one u32 per thread; `total` gets the block's sum.
template <int NT>
__device__ __forceinline__ u32 block_excl_sum(u32 v, u32 *sw, u32 &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u32 inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sw[w] = inc;
    __syncthreads();
    u32 off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) {
        off += (i < w) ? sw[i] : 0u;
        tot += sw[i];
    }
    __syncthreads();
    total = tot;
    return off + inc - v;
}

// The kernel's phases: the generator into a window, make-and-count, make.
// PG_SMALL_NOINLINE 1 calls one out-of-line copy of each instead of inlining
// them at every call site (a tuning build; it measured no faster).
#ifndef PG_SMALL_NOINLINE
#define PG_SMALL_NOINLINE 0
#endif
#if PG_SMALL_NOINLINE
#define PG_SMALL_FN __device__ __noinline__
#else
#define PG_SMALL_FN __device__ __forceinline__
#endif
// Generates b's moves into items[rel0 ..] (those inside [0, n), tagged);
// returns rel0 plus the number of moves.  PG_SMALL_GEN_SV: the generator's
// slider variant here.  Kogge-Stone fills (0): one thread generating on a
// fresh launch waits on every table lookup, and the fills need none; the
// initial position at depth 5 took 68 us with them against 74 us with the
// generator's default magic lookups (-1).
#ifndef PG_SMALL_GEN_SV
#define PG_SMALL_GEN_SV 0
#endif
template <int SV>
PG_SMALL_FN int small_gen(Board b, u32 *items, int rel0, u32 n, u32 tag)
{
    WindowSink sink{items, rel0, n, tag};
    gen_moves<SV, false, PG_SMALL_GEN_SV>(b, sink);
    return sink.rel;
}

template <int SV>
PG_SMALL_FN u32 small_make_count(Board parent, u32 mv, Board *child)
{
    const Board c = make_child<false>(parent, mv);
    if (child) *child = c;
    return count_moves<SV>(c);
}

template <int SV>
PG_SMALL_FN Board small_make(Board parent, u32 mv)
{
    return make_child<false>(parent, mv);
}

// Exclusive offsets of the counts c[0..n) (n <= MAX_LEGAL_MOVES) into
// off[0..n); returns their total.  Each thread scans SMALL_PER consecutive
// entries.
template <int NT>
__device__ __forceinline__ u32 small_scan(const u32 *c, u32 *off, u32 n, u32 *sw)
{
    constexpr int PER = (MAX_LEGAL_MOVES + NT - 1) / NT;
    const u32 t0 = threadIdx.x * PER;
    u32 v = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) v += (t0 + k < n) ? c[t0 + k] : 0u;
    u32 total;
    u32 base = block_excl_sum<NT>(v, sw, total);
#pragma unroll
    for (int k = 0; k < PER; k++)
        if (t0 + k < n) {
            off[t0 + k] = base;
            base += c[t0 + k];
        }
    __syncthreads();
    return total;
}

// listCap: subtree roots a CTA may list, at most SMALL_LIST_CAP.
template <int SV>
__global__ void __launch_bounds__(SMALL_NT, SMALL_MINB) k_small_tree(const u64 *__restrict__ pos48, int depth,
                                                                     u32 listCap, u64 *__restrict__ out,
                                                                     SmallState *S)
{
    __shared__ Board sB1[MAX_LEGAL_MOVES];  // the position's children (depth 5)
    __shared__ Board sX[MAX_LEGAL_MOVES];   // the current subtree root's children
    __shared__ u32 sM1[MAX_LEGAL_MOVES];    // the position's moves
    __shared__ u32 sMR[MAX_LEGAL_MOVES];    // the current subtree root's moves
    __shared__ u32 sC[MAX_LEGAL_MOVES];     // children's move counts
    __shared__ u32 sOff[MAX_LEGAL_MOVES];   // and their exclusive offsets
    __shared__ u32 swarp[SMALL_NT / 32];
    __shared__ u32 sN;
    __shared__ unsigned long long sSum[SMALL_NT / 32];
    __shared__ bool sLast;
    extern __shared__ __align__(16) u32 sdyn[];
    u32 *sList = sdyn;                   // depth 5: subtree roots as (child << 16) | move
    u32 *sItems = sdyn + SMALL_LIST_CAP;  // grandchildren as (child << 16) | move

    const int tid = threadIdx.x, lane = tid & 31;
    u64 p[6];
#pragma unroll
    for (int k = 0; k < 6; k++) p[k] = pos48[k];
    const Board root = from_pos48(p);
    const int r = depth >= 3 ? 3 : 2;
    const int pre = depth - r;  // plies from the position to the subtree roots: 0, 1 or 2
    u32 flags = validate_pos48(p) != 0 ? DERR_BAD_POSITION : 0u;
    u32 nRoots = 1;
    if (!flags && pre >= 1) {
        if (tid == 0) sN = (u32)small_gen<SV>(root, sM1, 0, MAX_LEGAL_MOVES, 0u);
        __syncthreads();
        const u32 n1 = sN;
        nRoots = n1;
        if (n1 > (u32)MAX_LEGAL_MOVES) flags = SMALL_OVERFLOW;
        if (!flags && pre == 2) {
            for (u32 t = tid; t < n1; t += SMALL_NT) sC[t] = small_make_count<SV>(root, sM1[t], &sB1[t]);
            __syncthreads();
            const u32 total = small_scan<SMALL_NT>(sC, sOff, n1, swarp);
            if (total > listCap) {
                flags = SMALL_OVERFLOW;
            } else {
                for (u32 t = tid; t < n1; t += SMALL_NT)
                    if (sC[t]) small_gen<SV>(sB1[t], sList, (int)sOff[t], listCap, t << 16);
                nRoots = total;
            }
        }
        __syncthreads();  // every thread has read sN and the lists before the loop rewrites them
    }

    unsigned long long acc = 0;
    for (u32 s = blockIdx.x; !flags && s < nRoots; s += gridDim.x) {
        Board R = root;
        if (pre == 1) R = small_make<SV>(root, sM1[s]);
        if (pre == 2) {
            const u32 e = sList[s];
            R = small_make<SV>(sB1[e >> 16], e & 0xFFFFu);
        }
        if (tid == 0) sN = (u32)small_gen<SV>(R, sMR, 0, MAX_LEGAL_MOVES, 0u);
        __syncthreads();
        const u32 nA = sN;
        if (nA > (u32)MAX_LEGAL_MOVES) {
            flags = SMALL_OVERFLOW;
            break;
        }
        for (u32 t = tid; t < nA; t += SMALL_NT) {
            const u32 c = small_make_count<SV>(R, sMR[t], &sX[t]);
            sC[t] = c;
            if (r == 2) acc += c;
        }
        __syncthreads();
        if (r == 2) continue;  // sMR, sC and sN are rewritten only after this barrier
        const u32 T = small_scan<SMALL_NT>(sC, sOff, nA, swarp);
        for (u32 w0 = 0; w0 < T; w0 += SMALL_WIN) {
            const u32 wn = min(SMALL_WIN, T - w0);
            for (u32 t = tid; t < nA; t += SMALL_NT) {
                const u32 c = sC[t], off = sOff[t];
                if (c && off + c > w0 && off < w0 + wn)
                    small_gen<SV>(sX[t], sItems, (int)((long long)off - (long long)w0), wn, t << 16);
            }
            __syncthreads();
            for (u32 j = tid; j < wn; j += SMALL_NT) {
                const u32 it = sItems[j];
                acc += small_make_count<SV>(sX[it >> 16], it & 0xFFFFu, nullptr);
            }
            __syncthreads();
        }
    }

    // per-CTA sum, then the last CTA to finish adds them up
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) sSum[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        unsigned long long t = 0;
#pragma unroll
        for (int i = 0; i < SMALL_NT / 32; i++) t += sSum[i];
        S->partial[blockIdx.x] = t;
        if (flags) atomicOr(&S->flagAcc, flags);
        __threadfence();
        sLast = atomicInc(&S->done, gridDim.x - 1) == gridDim.x - 1;
    }
    __syncthreads();
    if (!sLast) return;
    __threadfence();
    unsigned long long t = 0;
    for (u32 i = tid; i < gridDim.x; i += SMALL_NT) t += __ldcg(&S->partial[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sSum[tid >> 5] = t;
    __syncthreads();
    if (tid == 0) {
        unsigned long long sum = 0;
#pragma unroll
        for (int i = 0; i < SMALL_NT / 32; i++) sum += sSum[i];
        const u32 all = atomicExch(&S->flagAcc, 0u) | flags;
        S->count = all ? 0ull : sum;
        S->flags = all;
        if (!all) out[0] = sum;
    }
}

// ====================================================== transposition table
// Lockless table of 16-byte entries {verify ^ value, value} at the slot the
// slot key picks: a torn or foreign entry fails the XOR check (the
// reference's scheme, perft_bb.h:759-764, whose 128-bit hash is here two
// independent 64-bit hashes).  Both are Zobrist hashes of the side-relative
// board (two sets of 781 seeded keys: 12 piece kinds x 64 squares, 4 castling
// rights, 8 en-passant files, one spare) XOR a per-remaining-depth key, so
// one table holds every depth ("per-depth slots").  Perft is invariant under the
// colour mirror, so a position and its mirror may share an entry.
constexpr int ZOB_KEYS = 781;
constexpr int ZOB_DEPTH_KEYS = 32;
// Two independent key sets (x, y): the x hash picks the table slot and the
// de-duplication slot, the y hash verifies.  A verification key that shares
// no bits with the index keeps false hits at 2^-64 per probe; with one 64-bit
// hash doing both, only the bits above the index are checked, and searches
// with ~1e12 probes (perft 12 of the initial position) did see false hits.
__device__ ulonglong2 d_zobrist[ZOB_KEYS + ZOB_DEPTH_KEYS];

constexpr u32 ALIAS_HIT = 0xFFFFFFFFu;     // value came from the table
constexpr u32 ALIAS_NOSLOT = 0xFFFFFFFEu;  // not de-duplicated (set full)
constexpr u64 DEDUP_EMPTY = ~0ULL;
constexpr int DEDUP_MAX_PROBES = 64;

struct TTStats {
    unsigned long long probes, hits, aliases, stores;
};

__device__ __forceinline__ void zx(ulonglong2 &h, int k)
{
    const ulonglong2 z = __ldg(&d_zobrist[k]);
    h.x ^= z.x;
    h.y ^= z.y;
}

// Both Zobrist hashes of a side-relative board (one 16-byte key load per piece).
__device__ __forceinline__ ulonglong2 zobrist_rel(const Board &b)
{
    const u64 pawns = b.pawns & RANKS2TO7;
    const u64 occ = pawns | b.knights | b.bq | b.rq | b.kings;
    const u64 theirs = occ ^ b.mine;
    const u64 sets[6] = {pawns, b.knights, b.bq & ~b.rq, b.rq & ~b.bq, b.bq & b.rq, b.kings};
    ulonglong2 h = make_ulonglong2(0, 0);
#pragma unroll
    for (int pc = 0; pc < 6; pc++) {
        u64 m = sets[pc] & b.mine;
        while (m) {
            zx(h, pc * 64 + ctz(m));
            m &= m - 1;
        }
        u64 t = sets[pc] & theirs;
        while (t) {
            zx(h, (6 + pc) * 64 + ctz(t));
            t &= t - 1;
        }
    }
    const u32 st = (u32)(b.pawns & 0xFF);
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (st & (1u << k)) zx(h, 768 + k);
    if (st >> 4) zx(h, 772 + (st >> 4) - 1);
    return h;
}

// Block-aggregated increment of a statistics counter: warp ballots summed
// in shared memory, then one global atomic per block.  Per-warp atomics on
// the same few counters serialised in L2 and cost a large part of the table
// kernels' time.  Every thread of the block must call it.
__device__ __forceinline__ void count_stat(unsigned long long *ctr, bool hit)
{
    __shared__ unsigned sCount;
    if (threadIdx.x == 0) sCount = 0;
    __syncthreads();
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(&sCount, (unsigned)__popc(m));
    __syncthreads();
    if (threadIdx.x == 0 && sCount) atomicAdd(ctr, (unsigned long long)sCount);
}

// Hash every node, probe the table, and insert misses into the level's
// de-duplication set (lowest index wins).  Hits get their value and no
// children; their alias is ALIAS_HIT.  Misses keep the set slot in alias.
__global__ void __launch_bounds__(256) k_tt_probe(const u64 *__restrict__ planes, u64 stride, u64 n, int remaining,
                                                  bool probe, u64 keyMask, u32 *__restrict__ cnt,
                                                  u64 *__restrict__ hash, u64 *__restrict__ hash2,
                                                  unsigned long long *__restrict__ acc, u32 *__restrict__ alias,
                                                  const ulonglong2 *tt, u64 ttMask, u64 *__restrict__ dkey,
                                                  u32 *__restrict__ downer, u64 dMask, TTStats *ts)
{
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    bool hit = false;
    if (i < n) {
        const Board b = level_get(planes, stride, i);
        ulonglong2 z = zobrist_rel(b);
        zx(z, ZOB_KEYS + remaining);
        const u64 h = z.x & keyMask;  // slot key (table index, de-duplication set)
        const u64 g = z.y;            // verification key
        hash[i] = h;
        hash2[i] = g;
        acc[i] = 0;
        if (probe) {
            const ulonglong2 e = tt[h & ttMask];
            if ((e.x ^ e.y) == g) {
                hit = true;
                acc[i] = e.y;
                cnt[i] = 0;
                alias[i] = ALIAS_HIT;
            }
        }
        if (!hit) {
            u32 placed = ALIAS_NOSLOT;
            if (h != DEDUP_EMPTY) {
                u64 slot = (h * 0x9E3779B97F4A7C15ULL >> 17) & dMask;
                for (int k = 0; k < DEDUP_MAX_PROBES; k++) {
                    const unsigned long long old =
                        atomicCAS((unsigned long long *)&dkey[slot], (unsigned long long)DEDUP_EMPTY,
                                  (unsigned long long)h);
                    if (old == DEDUP_EMPTY || old == h) {
                        atomicMin(&downer[slot], (u32)i);
                        placed = (u32)slot;
                        break;
                    }
                    slot = (slot + 1) & dMask;
                }
            }
            alias[i] = placed;
        }
    }
    if (probe) {
        count_stat(&ts->probes, i < n);
        count_stat(&ts->hits, hit);
    }
}

// Turns set slots into owner indices; duplicates lose their children.  A
// node shares its owner's slot key; it is a duplicate only if the
// verification keys match too, otherwise it is searched on its own.
__global__ void __launch_bounds__(256) k_tt_dedup(u64 n, u32 *__restrict__ cnt, u32 *__restrict__ alias,
                                                  const u32 *__restrict__ downer, const u64 *__restrict__ hash2,
                                                  TTStats *ts)
{
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    bool dup = false;
    if (i < n) {
        const u32 a = alias[i];
        if (a != ALIAS_HIT && a != ALIAS_NOSLOT) {
            const u32 o = downer[a];
            if (o == (u32)i) {
                alias[i] = o;
            } else if (hash2[o] == hash2[i]) {
                alias[i] = o;
                cnt[i] = 0;
                dup = true;
            } else {
                alias[i] = ALIAS_NOSLOT;
            }
        }
    }
    count_stat(&ts->aliases, dup);
}

// After a level's subtrees are summed into acc: copy owners' values into
// their duplicates, store owners in the table, and add every value into the
// parent level (nodes are ordered by parent: segmented warp sums, then one
// atomic per parent run).  At level 0 the values go to the roots' results.
__global__ void __launch_bounds__(256) k_tt_finish(u64 n, bool store, const u64 *__restrict__ hash,
                                                   const u64 *__restrict__ hash2,
                                                   unsigned long long *__restrict__ acc, const u32 *__restrict__ alias,
                                                   const u32 *__restrict__ parent, unsigned long long *parentAcc,
                                                   ulonglong2 *tt, u64 ttMask, TTStats *ts)
{
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    unsigned long long v = 0;
    u32 key = 0xFFFFFFFFu;
    bool stored = false;
    if (i < n) {
        const u32 a = alias[i];
        v = acc[i];
        if (a != ALIAS_HIT && a != ALIAS_NOSLOT && a != (u32)i) {
            v = acc[a];  // the owner is final: its subtree finished before this kernel
        } else if (a != ALIAS_HIT && store) {
            tt[hash[i] & ttMask] = make_ulonglong2(hash2[i] ^ v, v);
            stored = true;
        }
        key = parent[i];
    }
    count_stat(&ts->stores, stored);
    if (!parentAcc) return;  // level 0: k_tt_roots writes the results
    // segmented inclusive sum over runs of equal parent within the warp
    unsigned long long sum = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, sum, o);
        const u32 ky = __shfl_up_sync(0xffffffffu, key, o);
        if (lane >= o && ky == key) sum += y;
    }
    const u32 knext = __shfl_down_sync(0xffffffffu, key, 1);
    const bool last = (lane == 31) || knext != key;
    if (i < n && last && key != 0xFFFFFFFFu) atomicAdd(&parentAcc[key], sum);
}

// Level 0 of a TT run: each root's value (own, owner's, or table's) is its result.
__global__ void k_tt_roots(u64 n, const unsigned long long *__restrict__ acc, const u32 *__restrict__ alias,
                           const u32 *__restrict__ root, unsigned long long *__restrict__ out)
{
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 a = alias[i];
    out[root[i]] = (a != ALIAS_HIT && a != ALIAS_NOSLOT && a != (u32)i) ? acc[a] : acc[i];
}

// ================================================================ host side
struct DeviceLevel {
    u64 *planes;
    u64 stride;
    u32 *cnt;
    u32 *root;  // root id (no TT) or parent index in the previous level (TT)
    u64 n;
    // transposition-table runs only
    u64 *hash = nullptr;   // slot key
    u64 *hash2 = nullptr;  // verification key
    unsigned long long *acc = nullptr;  // perft of each node's subtree
    u32 *alias = nullptr;               // owner index, ALIAS_HIT or ALIAS_NOSLOT
};

// Bytes of one TT level node: the plain node plus two hashes, subtree sum, alias,
// and the transient de-duplication set (at most 2.5 slots of 12 bytes per
// node; it is released before the scan, so this over-counts slightly).
constexpr u64 NODE_BYTES_TT = NODE_BYTES + 8 + 8 + 8 + 4 + 30;

class Engine {
public:
    int init(const perft_config &cfg);
    void shutdown();
    // trySmall: a single position of depth 2..5 tries the one-launch
    // small-tree kernel first (false when the caller already tried it)
    int run_batch(const u64 *dPos, const uint8_t *depths, u32 n, u64 *dOut, bool trySmall = true);
    // Host buffers: staged through engine-owned device buffers that persist
    // across calls (no per-call allocation; stable addresses let replayed
    // graphs be reused).
    int run_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out);
    u64 *ioPos = nullptr, *ioOut = nullptr;
    u32 ioCap = 0;

    perft_stats stats{};
    std::mutex mu;
    bool ready = false;
    std::string lastCudaError;

private:
    int device = 0;
    int nsm = 0;
    cudaStream_t stream = nullptr;
    char *arena = nullptr;
    u64 arenaCap = 0, arenaTop = 0, arenaPeak = 0;
    u32 *dCounter = nullptr;  // tile cursor
    u32 *dErr = nullptr;
    u64 *hPinned = nullptr;   // small read-backs
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int svExpand = SV_KOGGE, svLeaf = SV_KOGGE;
    int gridTile[2][SV_COUNT] = {};
    bool trace = false;  // PERFT_TRACE=1: one stderr line per tile launch

public:
    // Launch configuration per (ply kind, remaining depth of the parent level):
    // slider variant, largest tile (log2 items) and resident CTAs per SM.  The
    // count-only ply always has remaining depth 2; interior plies have 3..20
    // and use the entry of the nearest calibrated depth.
    struct TuneCfg {
        int sv = SV_KOGGE;
        int cap = TILE_CAP_LOG2;
        int ctas = 0;  // 0: as many as fit
        double ms = 0;  // calibration time of this key (median of the timed runs)
    };
    static constexpr int TUNE_MAX_R = 20;
    TuneCfg tuneTab[2][TUNE_MAX_R + 1];
    int tunedMaxR = 3;

private:
    bool tuning = false;  // autotune running: launch times accumulate per key
    double tuneAccMs[2][TUNE_MAX_R + 1] = {};
    const TuneCfg &cfg_for(int mode, int r) const
    {
        if (mode == MODE_LEAF) return tuneTab[MODE_LEAF][2];
        return tuneTab[MODE_EXPAND][std::max(3, std::min(r, tunedMaxR))];
    }
    int grid_for(int mode, const TuneCfg &c) const
    {
        const int occ = gridTile[mode][c.sv];
        return c.ctas > 0 ? std::min(occ, c.ctas * nsm) : occ;
    }
    int max_ctas(int mode, int sv) const { return std::max(1, gridTile[mode][sv] / std::max(1, nsm)); }
    void fill_tune(int svL, int svE)
    {
        for (int r = 0; r <= TUNE_MAX_R; r++) {
            tuneTab[MODE_LEAF][r] = TuneCfg{svL, TILE_CAP_LOG2, 0, 0};
            tuneTab[MODE_EXPAND][r] = TuneCfg{svE, TILE_CAP_LOG2, 0, 0};
        }
        tunedMaxR = 3;
    }

    void *alloc(u64 bytes)
    {
        const u64 a = (arenaTop + 255) & ~255ULL;
        if (a + bytes > arenaCap) return nullptr;
        arenaTop = a + bytes;
        arenaPeak = std::max(arenaPeak, arenaTop);
        return arena + a;
    }
    u64 arena_free() const { return arenaCap > arenaTop ? arenaCap - arenaTop : 0; }
    bool alloc_level(DeviceLevel &L, u64 n);
    int scan(const u32 *cnt, u64 n, int remaining, u64 *&scanOut, u32 *&tileFirst, u64 &total, int &capLog2);
    int launch_tile(int mode, int remaining, const DeviceLevel &parents, const u64 *pscan, const u32 *tileFirst,
                    int capLog2, u64 itemBase, u64 itemEnd, DeviceLevel *children, unsigned long long *rootCounts);
    // Roots that join the search at a given remaining depth: their ids (device
    // array) and count, indexed by depth.  A root of depth d enters the level
    // whose nodes have d plies left, behind that level's children.
    struct Joiners {
        const u64 *dPos = nullptr;
        const u32 *ids[21] = {};
        u32 n[21] = {};
    };
    int process_level(const DeviceLevel &L, int remaining, unsigned long long *rootCounts,
                      const Joiners *join = nullptr);
    int init_joiners(const Joiners &J, int depth, DeviceLevel &C, u64 at, unsigned long long *rootCounts);
    int process_level_tt(const DeviceLevel &L, int remaining, unsigned long long *parentAcc,
                         unsigned long long *rootOut);
    bool alloc_level_tt(DeviceLevel &L, u64 n);

public:
    // A long-lived block at the top of the arena (the server's memory);
    // per-call allocations stack above it.
    char *reserve_block(u64 bytes)
    {
        blockMark = arenaTop;
        char *p = (char *)alloc(bytes);
        if (!p) arenaTop = blockMark;
        return p;
    }
    void release_block() { arenaTop = blockMark; }
    u64 free_bytes() const { return arena_free(); }
    int device_id() const { return device; }
    int leaf_sliders() const { return svLeaf; }
    u64 blockMark = 0;
    // The transposition table as the server sees it (null table: none configured).
    struct TTView {
        ulonglong2 *table;
        u64 mask, keyMask;
    };
    TTView tt_view() const { return TTView{tt, ttMask, ttKeyMask}; }
    int tt_clear();
    void read_tt_stats()
    {
        TTStats t{};
        if (dTTStats && cudaMemcpy(&t, dTTStats, sizeof t, cudaMemcpyDeviceToHost) == cudaSuccess) {
            stats.tt_probes = t.probes;
            stats.tt_hits = t.hits;
            stats.tt_duplicates = t.aliases;
            stats.tt_stores = t.stores;
        }
        stats.tt_entries = tt ? ttMask + 1 : 0;
    }
    void zero_tt_stats()
    {
        if (dTTStats) cudaMemset(dTTStats, 0, sizeof(TTStats));
    }

private:
    ulonglong2 *tt = nullptr;
    u64 ttMask = 0;
    u64 ttKeyMask = ~0ULL;
    TTStats *dTTStats = nullptr;
    int ttMinDepth = 2;
    int check(cudaError_t e, const char *what);
    int sync_and_check_errors();
    int autotune(bool leaf, bool expand);

    // device-driven runs captured as CUDA graphs (small single-depth batches)
    struct DDGraph {
        int depth = 0;                // deepest root
        std::vector<uint8_t> depths;  // every root's depth (the graph's plan depends on the mix)
        u32 n = 0;
        const u64 *dPos = nullptr;
        u64 *dOut = nullptr;
        u64 top = 0;
        int svL = 0, svE = 0;
        bool overflowed = false;  // the plan did not fit: later calls go host-driven at once
        cudaEvent_t evLeaf0 = nullptr, evLeaf1 = nullptr;  // recorded around the count-only ply
        std::vector<double> predLv;  // predicted nodes per level (empty: no prediction)
        u64 otherLaunches = 0;       // root, scan and join kernels per replay
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        DevPlan *hTemplate = nullptr;  // pinned
        u32 *hIds = nullptr;           // pinned
        u64 *hFlags = nullptr;         // pinned: overflow, device error, leaf items
    };
    std::vector<DDGraph> ddCache;
    // one-launch small trees (k_small_tree)
    SmallState *dSmall = nullptr;
    int smallGrid = 0;
    bool smallEnabled = true;
    u32 smallListCap = SMALL_LIST_CAP;
    int run_small(const u64 *dPos, int depth, u64 *dOut, u64 *hOut, bool &handled);
    bool ddEnabled = true;
    bool ddForce = false;  // PERFT_DD_FORCE=1: skip the size estimate (tests the overflow fallback)
    double ddMaxBytes = DD_MAX_BYTES_DEFAULT;
    int ddGridScan = 0;
    int run_dd(const u64 *dPos, const uint8_t *depths, u32 n, u64 *dOut, bool &handled);
    int build_dd(DDGraph &G);
    void drop_dd();
};

int Engine::check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return PERFT_OK;
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    lastCudaError = buf;
    return e == cudaErrorMemoryAllocation ? PERFT_ERR_OUT_OF_MEMORY : PERFT_ERR_CUDA;
}

#define ENG_TRY(expr)                                   \
    do {                                                \
        int rc_ = check((expr), #expr);                 \
        if (rc_ != PERFT_OK) return rc_;                \
    } while (0)

constexpr size_t TILE_DYN_SMEM = sizeof(u32) * TILE_CAP;

// Allows the item list's dynamic shared memory on one instantiation and
// returns its resident-CTA grid (SMs x CTAs per SM).
template <int MODE, int SV>
int occupancy_grid(int nsm)
{
    cudaFuncSetAttribute(k_tile<MODE, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_DYN_SMEM);
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_tile<MODE, SV>, TILE_NT, TILE_DYN_SMEM) !=
            cudaSuccess ||
        perSm < 1)
        perSm = 1;
    return perSm * nsm;
}

template <int MODE>
void launch_tile_variant(int sv, int grid, cudaStream_t st, const TileParams &P)
{
    switch (sv) {
    case SV_MAGIC: k_tile<MODE, SV_MAGIC><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P); break;
    case SV_KOGGE_FMA: k_tile<MODE, SV_KOGGE_FMA><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P); break;
    case SV_KOGGE_SPLIT: k_tile<MODE, SV_KOGGE_SPLIT><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P); break;
    case SV_HYBRID: k_tile<MODE, SV_HYBRID><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P); break;
    default: k_tile<MODE, SV_KOGGE><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P); break;
    }
}

// A device-driven tile launch: the two graph variants (Kogge-Stone, split
// shifts) x the two parameter modes (constant bank for large plies, shared
// memory for small ones).
template <int MODE>
void launch_dd_tile(int sv, bool constParams, int grid, cudaStream_t st, const TileParams &P)
{
    const bool split = sv == SV_KOGGE_SPLIT;
    if (constParams && split) k_tile<MODE, SV_KOGGE_SPLIT, false, DD_CONST><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P);
    else if (constParams) k_tile<MODE, SV_KOGGE, false, DD_CONST><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P);
    else if (split) k_tile<MODE, SV_KOGGE_SPLIT, false, DD_SHARED><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P);
    else k_tile<MODE, SV_KOGGE, false, DD_SHARED><<<grid, TILE_NT, TILE_DYN_SMEM, st>>>(P);
}

const char *slider_name(int sv)
{
    switch (sv) {
    case SV_KOGGE: return "kogge";
    case SV_MAGIC: return "magic";
    case SV_KOGGE_FMA: return "kogge_fma";
    case SV_KOGGE_SPLIT: return "kogge_split";
    case SV_HYBRID: return "hybrid";
    default: return "?";
    }
}

int Engine::init(const perft_config &cfg)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return PERFT_ERR_NO_DEVICE;
    if (cfg.device < 0 || cfg.device >= ndev) return PERFT_ERR_INVALID_ARG;
    device = cfg.device;
    trace = getenv("PERFT_TRACE") && getenv("PERFT_TRACE")[0] == '1';
    ENG_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    ENG_TRY(cudaGetDeviceProperties(&prop, device));
    nsm = prop.multiProcessorCount;

    build_tables();
    ENG_TRY(cudaMemcpyToSymbol(d_tables, &h_tables, sizeof(Tables)));
    ENG_TRY(cudaMemcpyToSymbol(d_magic, h_magic, sizeof(h_magic)));
    u32 pow2[32];
    for (int k = 0; k < 32; k++) pow2[k] = 1u << k;
    ENG_TRY(cudaMemcpyToSymbol(c_pow2, pow2, sizeof pow2));

    // A blocking stream: it orders against the legacy default stream, where
    // callers (and torch) usually produce device-resident inputs.
    ENG_TRY(cudaStreamCreate(&stream));
    ENG_TRY(cudaEventCreate(&ev0));
    ENG_TRY(cudaEventCreate(&ev1));
    ENG_TRY(cudaMalloc(&dCounter, 64));
    ENG_TRY(cudaMalloc(&dErr, 64));
    ENG_TRY(cudaMallocHost(&hPinned, 64));

    // Zobrist keys (splitmix64 of the seed) and the transposition table
    {
        ulonglong2 keys[ZOB_KEYS + ZOB_DEPTH_KEYS];
        u64 x = cfg.zobrist_seed;
        auto next = [&x]() {
            x += 0x9E3779B97F4A7C15ULL;
            u64 z = x;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            return z ^ (z >> 31);
        };
        for (int k = 0; k < ZOB_KEYS + ZOB_DEPTH_KEYS; k++) keys[k].x = next();
        for (int k = 0; k < ZOB_KEYS + ZOB_DEPTH_KEYS; k++) keys[k].y = next();
        ENG_TRY(cudaMemcpyToSymbol(d_zobrist, keys, sizeof keys));
        // PERFT_TT_INDEX_KEY_BITS=b keeps only the low b bits of the slot key:
        // a test setting that makes different positions share table and
        // de-duplication slots, which the verification key must then tell apart
        ttKeyMask = ~0ULL;
        if (const char *kb = getenv("PERFT_TT_INDEX_KEY_BITS")) {
            const int bits = atoi(kb);
            if (bits >= 1 && bits < 64) ttKeyMask = (1ULL << bits) - 1;
        }
    }
    ENG_TRY(cudaMalloc(&dTTStats, sizeof(TTStats)));
    ENG_TRY(cudaMemset(dTTStats, 0, sizeof(TTStats)));
    if (cfg.tt_log2_entries > 0) {
        if (cfg.tt_log2_entries < 10 || cfg.tt_log2_entries > 34) return PERFT_ERR_INVALID_ARG;
        const u64 entries = 1ULL << cfg.tt_log2_entries;
        ENG_TRY(cudaMalloc(&tt, entries * sizeof(ulonglong2)));
        ENG_TRY(cudaMemset(tt, 0, entries * sizeof(ulonglong2)));
        ttMask = entries - 1;
    }

    size_t freeB = 0, totalB = 0;
    ENG_TRY(cudaMemGetInfo(&freeB, &totalB));
    u64 want = cfg.arena_bytes ? cfg.arena_bytes : (u64)(freeB * 0.85);
    if (want > freeB) return PERFT_ERR_OUT_OF_MEMORY;
    ENG_TRY(cudaMalloc(&arena, want));
    arenaCap = want;

    gridTile[MODE_EXPAND][SV_KOGGE] = occupancy_grid<MODE_EXPAND, SV_KOGGE>(nsm);
    gridTile[MODE_EXPAND][SV_MAGIC] = occupancy_grid<MODE_EXPAND, SV_MAGIC>(nsm);
    gridTile[MODE_EXPAND][SV_KOGGE_FMA] = occupancy_grid<MODE_EXPAND, SV_KOGGE_FMA>(nsm);
    gridTile[MODE_EXPAND][SV_KOGGE_SPLIT] = occupancy_grid<MODE_EXPAND, SV_KOGGE_SPLIT>(nsm);
    gridTile[MODE_LEAF][SV_KOGGE] = occupancy_grid<MODE_LEAF, SV_KOGGE>(nsm);
    gridTile[MODE_LEAF][SV_MAGIC] = occupancy_grid<MODE_LEAF, SV_MAGIC>(nsm);
    gridTile[MODE_LEAF][SV_KOGGE_FMA] = occupancy_grid<MODE_LEAF, SV_KOGGE_FMA>(nsm);
    gridTile[MODE_LEAF][SV_KOGGE_SPLIT] = occupancy_grid<MODE_LEAF, SV_KOGGE_SPLIT>(nsm);
    gridTile[MODE_EXPAND][SV_HYBRID] = occupancy_grid<MODE_EXPAND, SV_HYBRID>(nsm);
    gridTile[MODE_LEAF][SV_HYBRID] = occupancy_grid<MODE_LEAF, SV_HYBRID>(nsm);

    for (auto fn : {(const void *)k_tile<MODE_LEAF, SV_KOGGE, false, DD_CONST>,
                    (const void *)k_tile<MODE_LEAF, SV_KOGGE_SPLIT, false, DD_CONST>,
                    (const void *)k_tile<MODE_EXPAND, SV_KOGGE, false, DD_CONST>,
                    (const void *)k_tile<MODE_EXPAND, SV_KOGGE_SPLIT, false, DD_CONST>,
                    (const void *)k_tile<MODE_LEAF, SV_KOGGE, false, DD_SHARED>,
                    (const void *)k_tile<MODE_LEAF, SV_KOGGE_SPLIT, false, DD_SHARED>,
                    (const void *)k_tile<MODE_EXPAND, SV_KOGGE, false, DD_SHARED>,
                    (const void *)k_tile<MODE_EXPAND, SV_KOGGE_SPLIT, false, DD_SHARED>})
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_DYN_SMEM);
    ddGridScan = 4 * nsm;
    {
        ENG_TRY(cudaMalloc(&dSmall, sizeof(SmallState)));
        ENG_TRY(cudaMemset(dSmall, 0, sizeof(SmallState)));
        ENG_TRY(cudaFuncSetAttribute(k_small_tree<SV_KOGGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMALL_DYN_SMEM));
        int perSm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_small_tree<SV_KOGGE>, SMALL_NT, SMALL_DYN_SMEM) !=
                cudaSuccess ||
            perSm < 1)
            perSm = 1;
        smallGrid = std::min(SMALL_MAX_GRID, perSm * nsm);
        smallEnabled = !(getenv("PERFT_SMALL_TREE") && getenv("PERFT_SMALL_TREE")[0] == '0');
        // PERFT_SMALL_LIST_CAP=k lists at most k depth-5 subtree roots per CTA:
        // a test setting that sends ordinary positions down the fallback
        smallListCap = SMALL_LIST_CAP;
        if (const char *c = getenv("PERFT_SMALL_LIST_CAP")) {
            const long v = atol(c);
            if (v >= 1 && v <= (long)SMALL_LIST_CAP) smallListCap = (u32)v;
        }
    }
    ddEnabled = !(getenv("PERFT_NO_GRAPHS") && getenv("PERFT_NO_GRAPHS")[0] == '1');
    ddForce = getenv("PERFT_DD_FORCE") && getenv("PERFT_DD_FORCE")[0] == '1';
    ddMaxBytes = DD_MAX_BYTES_DEFAULT;
    if (const char *g = getenv("PERFT_DD_MAX_GB")) ddMaxBytes = atof(g) * (double)(1ull << 30);

    auto pick = [](int v) { return (v >= 0 && v < SV_COUNT) ? v : SV_KOGGE; };
    svExpand = pick(cfg.sliders_expand);
    svLeaf = pick(cfg.sliders_leaf);
    fill_tune(svLeaf, svExpand);
    ready = true;
    const bool tuneLeaf = cfg.sliders_leaf == PERFT_SLIDERS_AUTO;
    const bool tuneExpand = cfg.sliders_expand == PERFT_SLIDERS_AUTO;
    if (tuneLeaf || tuneExpand) {
        const int rc = autotune(tuneLeaf, tuneExpand);
        if (rc != PERFT_OK) {
            ready = false;
            return rc;
        }
    }
    memset(&stats, 0, sizeof stats);
    stats.sliders_expand = svExpand;
    stats.sliders_leaf = svLeaf;
    stats.arena_bytes = arenaCap;
    return PERFT_OK;
}

void Engine::shutdown()
{
    if (!ready) return;
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    drop_dd();
    if (ioPos) cudaFree(ioPos);
    if (ioOut) cudaFree(ioOut);
    ioPos = ioOut = nullptr;
    ioCap = 0;
    cudaFree(arena);
    if (tt) cudaFree(tt);
    tt = nullptr;
    ttMask = 0;
    if (dTTStats) cudaFree(dTTStats);
    dTTStats = nullptr;
    cudaFree(dCounter);
    cudaFree(dErr);
    if (dSmall) cudaFree(dSmall);
    dSmall = nullptr;
    cudaFreeHost(hPinned);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaStreamDestroy(stream);
    arena = nullptr;
    ready = false;
}

bool Engine::alloc_level(DeviceLevel &L, u64 n)
{
    L.n = n;
    L.stride = (n + 31) & ~31ULL;
    L.planes = (u64 *)alloc(6 * 8 * L.stride);
    L.cnt = (u32 *)alloc(4 * L.stride);
    L.root = (u32 *)alloc(4 * L.stride);
    return L.planes && L.cnt && L.root;
}

// `remaining`: remaining depth of the level scanned; its items go to the
// count-only ply when it is 2, to an interior ply otherwise.
int Engine::scan(const u32 *cnt, u64 n, int remaining, u64 *&scanOut, u32 *&tileFirst, u64 &total, int &capLog2)
{
    const u64 nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    const u64 maxTiles = (n * MAX_LEGAL_MOVES) / MAX_TILES_PER_NODE_DIV + 2;
    scanOut = (u64 *)alloc(8 * (n + 1));
    tileFirst = (u32 *)alloc(4 * maxTiles);
    u64 *bsum = (u64 *)alloc(8 * (nb + 1));
    if (!scanOut || !tileFirst || !bsum) return PERFT_ERR_OUT_OF_MEMORY;
    k_scan_reduce<<<(unsigned)nb, SCAN_NT, 0, stream>>>(cnt, n, bsum);
    k_scan_top<<<1, SCAN_TOP_NT, 0, stream>>>(bsum, nb, scanOut + n);
    ENG_TRY(cudaGetLastError());
    ENG_TRY(cudaMemcpyAsync(hPinned, scanOut + n, 8, cudaMemcpyDeviceToHost, stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    total = hPinned[0];
    // tile size: the tuned largest tile for this ply, made smaller while some
    // resident CTA would get no second tile
    const int mode = remaining == 2 ? MODE_LEAF : MODE_EXPAND;
    const TuneCfg &tc = cfg_for(mode, remaining);
    capLog2 = tc.cap;
    while (capLog2 > TILE_MIN_LOG2 && (total >> capLog2) < 2ull * grid_for(mode, tc)) capLog2--;
    k_scan_apply<<<(unsigned)nb, SCAN_NT, 0, stream>>>(cnt, n, bsum, scanOut, tileFirst, capLog2);
    stats.other_launches += 3;
    ENG_TRY(cudaGetLastError());
    return PERFT_OK;
}

int Engine::launch_tile(int mode, int remaining, const DeviceLevel &parents, const u64 *pscan, const u32 *tileFirst,
                        int capLog2, u64 itemBase, u64 itemEnd, DeviceLevel *children,
                        unsigned long long *rootCounts)
{
    TileParams P;
    memset(&P, 0, sizeof P);
    P.ppl = parents.planes;
    P.pstride = parents.stride;
    P.pscan = pscan;
    P.proot = parents.root;
    P.nParents = parents.n;
    P.tileFirst = tileFirst;
    P.itemBase = itemBase;
    P.itemEnd = itemEnd;
    P.capLog2 = capLog2;
    P.tileCounter = dCounter;
    if (children) {
        P.cpl = children->planes;
        P.cstride = children->stride;
        P.ccnt = children->cnt;
        P.croot = children->root;
    }
    P.rootCounts = rootCounts;
    P.err = dErr;

    const u64 nTiles = (itemEnd - itemBase + (1ull << capLog2) - 1) >> capLog2;
    const TuneCfg &tc = cfg_for(mode, remaining);
    const int sv = tc.sv;
    const int grid = (int)std::min<u64>((u64)grid_for(mode, tc), nTiles);
    ENG_TRY(cudaMemsetAsync(dCounter, 0, 4, stream));
    ENG_TRY(cudaEventRecord(ev0, stream));
    if (mode == MODE_LEAF) launch_tile_variant<MODE_LEAF>(sv, grid, stream, P);
    else launch_tile_variant<MODE_EXPAND>(sv, grid, stream, P);
    ENG_TRY(cudaGetLastError());
    ENG_TRY(cudaEventRecord(ev1, stream));
    ENG_TRY(cudaEventSynchronize(ev1));
    float ms = 0.f;
    ENG_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
    if (trace)
        fprintf(stderr, "perft-trace %s sv=%s parents=%llu items=%llu..%llu grid=%d ms=%.4f\n",
                mode == MODE_LEAF ? "leaf" : "expand", slider_name(sv), (unsigned long long)parents.n,
                (unsigned long long)itemBase, (unsigned long long)itemEnd, grid, ms);
    if (tuning) tuneAccMs[mode][mode == MODE_LEAF ? 2 : std::min(remaining, (int)TUNE_MAX_R)] += ms;
    if (mode == MODE_LEAF) {
        stats.leaf_launches++;
        stats.leaf_items += itemEnd - itemBase;
        stats.leaf_parents += parents.n;
        stats.leaf_ms += ms;
    } else {
        stats.expand_launches++;
        stats.expand_items += itemEnd - itemBase;
        stats.expand_ms += ms;
    }
    return PERFT_OK;
}

// L holds the nodes of one level, all with `remaining` plies left (>= 2).
// Writes the roots that join at remaining depth `depth` into C from index `at`.
int Engine::init_joiners(const Joiners &J, int depth, DeviceLevel &C, u64 at, unsigned long long *rootCounts)
{
    const u32 nj = J.n[depth];
    if (!nj) return PERFT_OK;
    k_init_roots<<<(nj + 127) / 128, 128, 0, stream>>>(J.dPos, J.ids[depth], nj, C.planes + 2 * at, C.stride,
                                                        C.cnt + at, C.root + at, depth, rootCounts, dErr);
    stats.other_launches++;
    return check(cudaGetLastError(), "k_init_roots");
}

// L holds the nodes of one level, all with `remaining` plies left (>= 2).
// With `join`, the roots of depth remaining - 1 are appended to the children
// (to the last chunk when the children are chunked), so every depth group of
// a batch shares one launch per ply: the deepest roots start the search and
// shallower ones join the level whose remaining depth equals theirs.
int Engine::process_level(const DeviceLevel &L, int remaining, unsigned long long *rootCounts, const Joiners *join)
{
    const u32 nJoin = (join && remaining - 1 >= 2) ? join->n[remaining - 1] : 0;
    if (L.n == 0 && nJoin == 0) return PERFT_OK;
    const u64 mark = arenaTop;
    u64 *pscan = nullptr;
    u32 *tileFirst = nullptr;
    u64 total = 0;
    int capLog2 = TILE_CAP_LOG2;
    int rc = L.n ? scan(L.cnt, L.n, remaining, pscan, tileFirst, total, capLog2) : PERFT_OK;
    if (rc != PERFT_OK) return rc;
    if (remaining == 2) {
        if (total) rc = launch_tile(MODE_LEAF, 2, L, pscan, tileFirst, capLog2, 0, total, nullptr, rootCounts);
        arenaTop = mark;
        return rc;
    }
    if (total == 0 && nJoin == 0) {
        arenaTop = mark;
        return PERFT_OK;
    }
    // interior ply: children fit whole, or in tile-aligned chunks
    const u64 slack = std::min<u64>(64ull << 20, arenaCap / 16);
    const u64 freeB = arena_free() > slack ? arena_free() - slack : 0;
    u64 budgetNodes = freeB / NODE_BYTES;
    if (remaining > 3) budgetNodes /= 2;  // leave room for the plies below
    budgetNodes = budgetNodes > nJoin ? budgetNodes - nJoin : 0;
    // whole level when it fits; otherwise tile-aligned chunks
    u64 chunk = total <= budgetNodes ? total : (budgetNodes & ~(u64)(TILE_CAP - 1));
    if (chunk == 0 && total) return PERFT_ERR_OUT_OF_MEMORY;
    if (chunk < total) stats.chunked_levels++;
    const u64 nChunks = total ? (total + chunk - 1) / chunk : 1;
    for (u64 k = 0; k < nChunks; k++) {
        const u64 lo = k * chunk, hi = std::min(total, lo + chunk);
        const bool last = k + 1 == nChunks;
        const u64 cm = arenaTop;
        DeviceLevel C;
        if (!alloc_level(C, (hi - lo) + (last ? nJoin : 0))) return PERFT_ERR_OUT_OF_MEMORY;
        if (hi > lo) {
            rc = launch_tile(MODE_EXPAND, remaining, L, pscan, tileFirst, capLog2, lo, hi, &C, nullptr);
            if (rc != PERFT_OK) return rc;
        }
        if (last && nJoin) {
            rc = init_joiners(*join, remaining - 1, C, hi - lo, rootCounts);
            if (rc != PERFT_OK) return rc;
        }
        rc = process_level(C, remaining - 1, rootCounts, join);
        if (rc != PERFT_OK) return rc;
        arenaTop = cm;
    }
    arenaTop = mark;
    return PERFT_OK;
}

// Per-depth autotuner.  A seeded calibration batch (32 playouts of 10-30
// plies at depth 6: interior plies with remaining depth 6..3, then the
// count-only ply) is run under candidate launch configurations, one warm-up
// and three timed runs each; every tile launch's CUDA-event time is charged
// to its (ply kind, remaining depth) key, and each key keeps the median of
// its three runs.  Coordinate search, every key at once:
//   1. slider variant (all five), largest tiles, all resident CTAs;
//   2. largest tile 2^13 / 2^12 / 2^11 items with each key's variant;
//   3. resident CTAs per SM: all that fit, or one fewer.
// A candidate replaces a key's current choice only when it is more than 1%
// faster, so near-ties resolve to the same (earlier) choice on every run.
// These are the reference's compile-time knobs (switches.h:13-26: block size,
// memory) chosen per depth on the device at hand.  Results are kept per
// device for the life of the process (PERFT_RETUNE=1 times again).
int Engine::autotune(bool leaf, bool expand)
{
    struct Cached {
        TuneCfg tab[2][TUNE_MAX_R + 1];
        int maxR;
    };
    static std::mutex cacheMu;
    static std::map<std::pair<int, int>, Cached> cache;
    const std::pair<int, int> key{device, (leaf ? 2 : 0) | (expand ? 1 : 0)};
    const bool retune = getenv("PERFT_RETUNE") && getenv("PERFT_RETUNE")[0] == '1';
    auto adopt = [&]() {
        svLeaf = tuneTab[MODE_LEAF][2].sv;
        svExpand = tuneTab[MODE_EXPAND][3].sv;
    };
    {
        std::lock_guard<std::mutex> lk(cacheMu);
        auto it = cache.find(key);
        if (!retune && it != cache.end()) {
            for (int m = 0; m < 2; m++) {
                for (int r = 0; r <= TUNE_MAX_R; r++) {
                    // a mode that is not tuned keeps the caller's variant
                    if ((m == MODE_LEAF && !leaf) || (m == MODE_EXPAND && !expand)) continue;
                    tuneTab[m][r] = it->second.tab[m][r];
                }
            }
            tunedMaxR = it->second.maxR;
            adopt();
            return PERFT_OK;
        }
    }

    constexpr u32 N = 32;
    constexpr int CAL_DEPTH = 6;
    std::vector<perft_pos48> pos(N);
    int rc = perft_random_playouts(0xA070707EULL, N, 10, 30, pos.data());
    if (rc != PERFT_OK) return rc;
    std::vector<uint8_t> depths(N, CAL_DEPTH);
    const u64 mark = arenaTop;
    u64 *dPos = (u64 *)alloc(48ull * N);
    u64 *dOut = (u64 *)alloc(8ull * N);
    if (!dPos || !dOut) return PERFT_ERR_OUT_OF_MEMORY;
    ENG_TRY(cudaMemcpyAsync(dPos, pos.data(), 48ull * N, cudaMemcpyHostToDevice, stream));
    ulonglong2 *keepTT = tt;
    tt = nullptr;  // time the kernels, not table hits
    const bool keepDD = ddEnabled;
    ddEnabled = false;  // the host-driven path times each launch
    struct Restore {
        Engine &e;
        ulonglong2 *t;
        bool dd;
        u64 mark;
        ~Restore()
        {
            e.tt = t;
            e.ddEnabled = dd;
            e.tuning = false;
            e.arenaTop = mark;
        }
    } restore{*this, keepTT, keepDD, mark};
    tunedMaxR = CAL_DEPTH;

    // median over the timed runs of each key's time under the current table
    double med[2][TUNE_MAX_R + 1];
    auto measure = [&]() -> int {
        std::vector<double> reps[2][TUNE_MAX_R + 1];
        for (int rep = 0; rep < 4; rep++) {
            memset(tuneAccMs, 0, sizeof tuneAccMs);
            tuning = true;
            const perft_stats keep = stats;
            const int r = run_batch(dPos, depths.data(), N, dOut);
            stats = keep;  // calibration runs stay out of the statistics
            tuning = false;
            if (r != PERFT_OK) return r;
            if (rep == 0) continue;  // warms caches and clocks
            for (int m = 0; m < 2; m++)
                for (int k = 0; k <= TUNE_MAX_R; k++) reps[m][k].push_back(tuneAccMs[m][k]);
        }
        for (int m = 0; m < 2; m++)
            for (int k = 0; k <= TUNE_MAX_R; k++) {
                std::sort(reps[m][k].begin(), reps[m][k].end());
                med[m][k] = reps[m][k][reps[m][k].size() / 2];
            }
        return PERFT_OK;
    };
    auto keys = [&](auto fn) {  // every tuned (mode, r) key of the calibration
        if (leaf) fn(MODE_LEAF, 2);
        if (expand)
            for (int r = 3; r <= CAL_DEPTH; r++) fn(MODE_EXPAND, r);
    };
    double best[2][TUNE_MAX_R + 1];
    TuneCfg chosen[2][TUNE_MAX_R + 1];
    auto apply = [&](int m, int r, const TuneCfg &c) {
        if (m == MODE_LEAF) {
            for (int k = 0; k <= TUNE_MAX_R; k++) tuneTab[MODE_LEAF][k] = c;
        } else {
            tuneTab[MODE_EXPAND][r] = c;
            if (r == 3)
                for (int k = 0; k < 3; k++) tuneTab[MODE_EXPAND][k] = c;
            if (r == CAL_DEPTH)
                for (int k = CAL_DEPTH + 1; k <= TUNE_MAX_R; k++) tuneTab[MODE_EXPAND][k] = c;
        }
    };
    // stage 1: slider variant
    for (int v = 0; v < SV_COUNT; v++) {
        keys([&](int m, int r) { apply(m, r, TuneCfg{v, TILE_CAP_LOG2, 0, 0}); });
        if ((rc = measure()) != PERFT_OK) return rc;
        keys([&](int m, int r) {
            if (v == 0 || med[m][r] < 0.99 * best[m][r]) {
                best[m][r] = med[m][r];
                chosen[m][r] = TuneCfg{v, TILE_CAP_LOG2, 0, med[m][r]};
            }
        });
    }
    // stage 2: largest tile
    for (int cap = TILE_CAP_LOG2 - 1; cap >= TILE_CAP_LOG2 - 2 && cap >= TILE_MIN_LOG2; cap--) {
        keys([&](int m, int r) { apply(m, r, TuneCfg{chosen[m][r].sv, cap, 0, 0}); });
        if ((rc = measure()) != PERFT_OK) return rc;
        keys([&](int m, int r) {
            if (med[m][r] < 0.99 * best[m][r]) {
                best[m][r] = med[m][r];
                chosen[m][r] = TuneCfg{chosen[m][r].sv, cap, 0, med[m][r]};
            }
        });
    }
    // stage 3: one resident CTA per SM fewer
    keys([&](int m, int r) {
        const TuneCfg &c = chosen[m][r];
        apply(m, r, TuneCfg{c.sv, c.cap, std::max(1, max_ctas(m, c.sv) - 1), 0});
    });
    if ((rc = measure()) != PERFT_OK) return rc;
    keys([&](int m, int r) {
        if (med[m][r] < 0.99 * best[m][r]) {
            best[m][r] = med[m][r];
            chosen[m][r] = TuneCfg{chosen[m][r].sv, chosen[m][r].cap, std::max(1, max_ctas(m, chosen[m][r].sv) - 1),
                                   med[m][r]};
        }
    });
    keys([&](int m, int r) { apply(m, r, chosen[m][r]); });
    adopt();
    {
        std::lock_guard<std::mutex> lk(cacheMu);
        Cached &c = cache[key];
        memcpy(c.tab, tuneTab, sizeof tuneTab);
        c.maxR = tunedMaxR;
    }
    return PERFT_OK;
}

bool Engine::alloc_level_tt(DeviceLevel &L, u64 n)
{
    if (!alloc_level(L, n)) return false;
    L.hash = (u64 *)alloc(8 * L.stride);
    L.hash2 = (u64 *)alloc(8 * L.stride);
    L.acc = (unsigned long long *)alloc(8 * L.stride);
    L.alias = (u32 *)alloc(4 * L.stride);
    return L.hash && L.hash2 && L.acc && L.alias;
}

int Engine::tt_clear()
{
    if (tt) ENG_TRY(cudaMemsetAsync(tt, 0, (ttMask + 1) * sizeof(ulonglong2), stream));
    ENG_TRY(cudaMemsetAsync(dTTStats, 0, sizeof(TTStats), stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    return PERFT_OK;
}

// Transposition-table version of process_level.  Every node of L (remaining
// plies `remaining`) is hashed and probed; hits and same-level duplicates
// are not expanded.  Subtree sums accumulate in L.acc: directly from the
// count-only last ply, or from the child levels' finish pass.  When L is
// done, owners are stored, duplicates copy their owner's value, and the
// values are added into parentAcc (or written to the roots' results).
int Engine::process_level_tt(const DeviceLevel &L, int remaining, unsigned long long *parentAcc,
                             unsigned long long *rootOut)
{
    if (L.n == 0) return PERFT_OK;
    const u64 mark = arenaTop;
    const unsigned nb = (unsigned)((L.n + 255) / 256);
    const bool useTT = remaining >= ttMinDepth;

    u64 dsize = 1024;
    while (dsize < L.n + L.n / 4) dsize <<= 1;  // load <= 80%; unplaced nodes are simply not de-duplicated
    u64 *dkey = (u64 *)alloc(8 * dsize);
    u32 *downer = (u32 *)alloc(4 * dsize);
    if (!dkey || !downer) return PERFT_ERR_OUT_OF_MEMORY;
    ENG_TRY(cudaMemsetAsync(dkey, 0xFF, 8 * dsize, stream));
    ENG_TRY(cudaMemsetAsync(downer, 0xFF, 4 * dsize, stream));
    k_tt_probe<<<nb, 256, 0, stream>>>(L.planes, L.stride, L.n, remaining, useTT, ttKeyMask, L.cnt, L.hash, L.hash2,
                                       L.acc, L.alias,
                                       tt, ttMask, dkey, downer, dsize - 1, dTTStats);
    k_tt_dedup<<<nb, 256, 0, stream>>>(L.n, L.cnt, L.alias, downer, L.hash2, dTTStats);
    stats.other_launches += 2;
    ENG_TRY(cudaGetLastError());
    arenaTop = mark;  // the de-duplication set is no longer needed

    u64 *pscan = nullptr;
    u32 *tileFirst = nullptr;
    u64 total = 0;
    int capLog2 = TILE_CAP_LOG2;
    int rc = scan(L.cnt, L.n, remaining, pscan, tileFirst, total, capLog2);
    if (rc != PERFT_OK) return rc;
    DeviceLevel self = L;
    self.root = nullptr;  // tile sums and child links point at the parent itself
    if (total > 0) {
        if (remaining == 2) {
            rc = launch_tile(MODE_LEAF, 2, self, pscan, tileFirst, capLog2, 0, total, nullptr, L.acc);
            if (rc != PERFT_OK) return rc;
        } else {
            const u64 slack = std::min<u64>(64ull << 20, arenaCap / 16);
            const u64 freeB = arena_free() > slack ? arena_free() - slack : 0;
            u64 budgetNodes = freeB / NODE_BYTES_TT;
            if (remaining > 3) budgetNodes /= 2;
            const u64 chunk = total <= budgetNodes ? total : (budgetNodes & ~(u64)(TILE_CAP - 1));
            if (chunk == 0) return PERFT_ERR_OUT_OF_MEMORY;
            if (chunk < total) stats.chunked_levels++;
            for (u64 lo = 0; lo < total; lo += chunk) {
                const u64 hi = std::min(total, lo + chunk);
                const u64 cm = arenaTop;
                DeviceLevel C;
                if (!alloc_level_tt(C, hi - lo)) return PERFT_ERR_OUT_OF_MEMORY;
                rc = launch_tile(MODE_EXPAND, remaining, self, pscan, tileFirst, capLog2, lo, hi, &C, nullptr);
                if (rc != PERFT_OK) return rc;
                rc = process_level_tt(C, remaining - 1, L.acc, nullptr);
                if (rc != PERFT_OK) return rc;
                arenaTop = cm;
            }
        }
    }
    arenaTop = mark;
    k_tt_finish<<<nb, 256, 0, stream>>>(L.n, useTT && tt != nullptr, L.hash, L.hash2, L.acc, L.alias, L.root,
                                        parentAcc, tt,
                                        ttMask, dTTStats);
    stats.other_launches++;
    if (rootOut) {
        k_tt_roots<<<nb, 256, 0, stream>>>(L.n, L.acc, L.alias, L.root, rootOut);
        stats.other_launches++;
    }
    ENG_TRY(cudaGetLastError());
    return PERFT_OK;
}

void Engine::drop_dd()
{
    for (DDGraph &G : ddCache) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        if (G.graph) cudaGraphDestroy(G.graph);
        cudaFreeHost(G.hTemplate);
        cudaFreeHost(G.hIds);
        cudaFreeHost(G.hFlags);
        if (G.evLeaf0) cudaEventDestroy(G.evLeaf0);
        if (G.evLeaf1) cudaEventDestroy(G.evLeaf1);
    }
    ddCache.clear();
}

// Captures one device-driven perft of G.n roots of any depth mix.  The
// deepest roots form level 0; a root of depth d joins level G.depth - d
// (behind that level's children), so every ply of the whole batch is one
// scan and one tile launch.  Roots of depth 0 and 1 are answered by
// k_init_roots.  Every buffer the graph reads is re-initialised inside it
// (plan, root ids, outputs), so the region above the arena top may be reused
// by other calls between replays.
int Engine::build_dd(DDGraph &G)
{
    const u64 n = G.n;
    const int d = G.depth;
    std::vector<u32> order;
    order.reserve(n);
    u32 nAt[DD_MAX_LEVELS + 2] = {};
    u64 offAt[DD_MAX_LEVELS + 2] = {};
    for (int dd = d; dd >= 0; dd--) {
        offAt[dd] = order.size();
        for (u32 i = 0; i < n; i++)
            if (G.depths[i] == dd) order.push_back(i);
        nAt[dd] = (u32)(order.size() - offAt[dd]);
    }
    const u64 off0 = (arenaTop + 255) & ~255ULL;
    char *base = arena + off0;
    const u64 cap = arenaCap - off0;
    u64 bump = 0;
    auto place = [&](u64 bytes) -> char * {
        const u64 a = (bump + 255) & ~255ULL;
        bump = a + bytes;
        return base + a;
    };
    DevPlan *dPlan = (DevPlan *)place(sizeof(DevPlan));
    u32 *dIds = (u32 *)place(4 * n);
    const u64 n0 = nAt[d];
    LevelDesc L0{};
    L0.n = n0;
    L0.nChild = 0;
    L0.stride = (n0 + 31) & ~31ULL;
    L0.planes = (u64 *)place(48 * L0.stride);
    L0.cnt = (u32 *)place(4 * L0.stride);
    L0.root = (u32 *)place(4 * L0.stride);
    L0.pscan = (u64 *)place(8 * (n0 + 1));
    L0.tileFirst = (u32 *)place(4 * ((n0 * MAX_LEGAL_MOVES) / MAX_TILES_PER_NODE_DIV + 2));
    L0.bsum = (u64 *)place(8 * ((n0 + SCAN_CHUNK - 1) / SCAN_CHUNK + 1));
    // scratch level for the roots of depth 0 and 1 (counts only)
    const u64 nShallow = std::max<u64>(nAt[0], nAt[1]);
    const u64 sStride = (nShallow + 31) & ~31ULL;
    u64 *sPlanes = (u64 *)place(48 * std::max<u64>(sStride, 32));
    u32 *sCnt = (u32 *)place(4 * std::max<u64>(sStride, 32));
    u32 *sRoot = (u32 *)place(4 * std::max<u64>(sStride, 32));
    if (bump > cap) return PERFT_ERR_OUT_OF_MEMORY;

    ENG_TRY(cudaMallocHost(&G.hTemplate, sizeof(DevPlan)));
    ENG_TRY(cudaMallocHost(&G.hIds, 4 * n));
    ENG_TRY(cudaMallocHost(&G.hFlags, 64));
    ENG_TRY(cudaEventCreate(&G.evLeaf0));
    ENG_TRY(cudaEventCreate(&G.evLeaf1));
    memset(G.hTemplate, 0, sizeof(DevPlan));
    G.hTemplate->base = base;
    G.hTemplate->cap = cap;
    G.hTemplate->bump = bump;
    G.hTemplate->tileTarget = 2 * gridTile[MODE_LEAF][G.svL];
    G.hTemplate->tileCounter = dCounter;
    G.hTemplate->lv[0] = L0;
    for (int dd = 2; dd < d; dd++) {
        G.hTemplate->joinN[d - dd] = nAt[dd];
        G.hTemplate->joinIds[d - dd] = dIds + offAt[dd];
    }
    // per ply: the tuned variant (one of the two graph instantiations) and largest tile
    auto ddSv = [](int v) { return (v == SV_KOGGE || v == SV_KOGGE_SPLIT) ? v : (int)SV_KOGGE; };
    int lvSv[DD_MAX_LEVELS] = {}, lvGrid[DD_MAX_LEVELS] = {};
    for (int lv = 0; lv <= d - 2; lv++) {
        const int r = d - lv, mode = r == 2 ? MODE_LEAF : MODE_EXPAND;
        const bool last = lv == d - 2;
        TuneCfg c = cfg_for(mode, r);
        c.sv = ddSv(c.sv);
        lvSv[lv] = c.sv;
        lvGrid[lv] = grid_for(mode, c);
        G.hTemplate->capMax[lv] = c.cap;
        TileParams &T = G.hTemplate->tp[lv];  // the scan fills the level fields on the device
        T.tileCounter = dCounter;
        T.rootCounts = (unsigned long long *)G.dOut;
        T.err = dErr;
        // A ply predicted to have few tiles gets a grid of four CTAs per
        // predicted tile (at least 8) instead of one CTA per resident slot:
        // the tile kernel is persistent, so any grid is correct, and the
        // CTAs that would find no tile cost launch and exit time.
        if ((int)G.predLv.size() > lv + 1) {
            const double items = last ? G.predLv[lv] * 32.0 : G.predLv[lv + 1];
            const double tiles = items / (double)(1u << TILE_MIN_LOG2) + 1.0;
            if (4.0 * tiles < (double)lvGrid[lv]) lvGrid[lv] = std::max(8, (int)(4.0 * tiles));
        }
    }
    memcpy(G.hIds, order.data(), 4 * n);

    ENG_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(dPlan, G.hTemplate, sizeof(DevPlan), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(dIds, G.hIds, 4 * n, cudaMemcpyHostToDevice, stream);
    cudaMemsetAsync(G.dOut, 0, 8 * n, stream);
    cudaMemsetAsync(dErr, 0, 4, stream);
    G.otherLaunches = (nAt[0] ? 1 : 0) + (nAt[1] ? 1 : 0) + (d >= 2 ? 1 : 0);
    for (int dd = 0; dd <= 1; dd++)
        if (nAt[dd])
            k_init_roots<<<(nAt[dd] + 127) / 128, 128, 0, stream>>>(G.dPos, dIds + offAt[dd], nAt[dd], sPlanes,
                                                                   sStride, sCnt, sRoot, dd,
                                                                   (unsigned long long *)G.dOut, dErr);
    if (d >= 2)
        k_init_roots<<<(unsigned)((n0 + 127) / 128), 128, 0, stream>>>(G.dPos, dIds + offAt[d], (u32)n0,
                                                                      L0.planes, L0.stride, L0.cnt, L0.root, d,
                                                                      (unsigned long long *)G.dOut, dErr);
    for (int lv = 0; lv <= d - 2; lv++) {
        const int last = lv == d - 2;
        // levels predicted small take one single-block scan launch instead of three
        if ((int)G.predLv.size() > lv && G.predLv[lv] <= 32768.0) {
            k_dd_scan_small<<<1, 1024, 0, stream>>>(dPlan, lv, last);
            G.otherLaunches += 1;
        } else {
            // grid-stride scans: large predicted levels get up to one block
            // per chunk (64 per SM at most), like the host-driven scan
            int sg = ddGridScan;
            if ((int)G.predLv.size() > lv)
                sg = (int)std::min<double>(64.0 * nsm, std::max<double>(ddGridScan, G.predLv[lv] / SCAN_CHUNK));
            k_dd_scan_reduce<<<sg, SCAN_NT, 0, stream>>>(dPlan, lv);
            G.otherLaunches += 3;
            k_dd_scan_top<<<1, SCAN_TOP_NT, 0, stream>>>(dPlan, lv, last);
            k_dd_scan_apply<<<sg, SCAN_NT, 0, stream>>>(dPlan, lv);
        }
        // (the scan reset the tile cursor)
        // Large plies read their launch parameters (completed by the scan)
        // from the constant bank, copied there by a copy node; small ones
        // from the plan, through shared memory (no copy node).
        const bool big = !((int)G.predLv.size() > lv + 1 &&
                           (last ? G.predLv[lv] * 32.0 : G.predLv[lv + 1]) < DD_CONST_MIN_ITEMS);
        if (big)
            cudaMemcpyToSymbolAsync(c_ddTile, &dPlan->tp[lv], sizeof(TileParams), 0, cudaMemcpyDeviceToDevice,
                                    stream);
        TileParams P;
        memset(&P, 0, sizeof P);
        P.planEntry = &dPlan->tp[lv];
        const int sv = lvSv[lv];
        const int grid = lvGrid[lv];
        if (last) {
            // external records: event record nodes in the graph (a plain
            // record during capture only orders the capture)
            cudaEventRecordWithFlags(G.evLeaf0, stream, cudaEventRecordExternal);
            launch_dd_tile<MODE_LEAF>(sv, big, grid, stream, P);
            cudaEventRecordWithFlags(G.evLeaf1, stream, cudaEventRecordExternal);
        } else {
            launch_dd_tile<MODE_EXPAND>(sv, big, grid, stream, P);
            const u32 nj = G.hTemplate->joinN[lv + 1];
            if (nj) {
                k_dd_join<<<(nj + 127) / 128, 128, 0, stream>>>(dPlan, lv + 1, G.dPos, dErr);
                G.otherLaunches += 1;
            }
        }
    }
    cudaMemcpyAsync(&G.hFlags[0], &dPlan->overflow, 4, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&G.hFlags[1], dErr, 4, cudaMemcpyDeviceToHost, stream);
    if (d >= 2) {
        cudaMemcpyAsync(&G.hFlags[2], &dPlan->lv[d - 2].total, 8, cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(&G.hFlags[3], &dPlan->lv[d - 2].n, 8, cudaMemcpyDeviceToHost, stream);
    }
    const cudaError_t ce = cudaStreamEndCapture(stream, &G.graph);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return check(ce, "capture of the device-driven perft");
    }
    ENG_TRY(cudaGraphInstantiate(&G.exec, G.graph, 0));
    return PERFT_OK;
}

// Batches whose predicted tree fits the arena run as one replayed graph,
// whatever their depth mix: the launch sequence is fixed and the sizes live
// on the device, so the host only waits once.  The prediction charges each
// root its own move count times 35 per further ply, 72 bytes per node of the
// last materialised ply (planes, count, root, scan entry, tile index) and of
// the plies above it, against 80% of the free arena.  `handled` stays false
// when the batch is not eligible or the device plan overflowed; the caller
// then runs the host-driven path.
int Engine::run_dd(const u64 *dPos, const uint8_t *depths, u32 n, u64 *dOut, bool &handled)
{
    handled = false;
    if (!ddEnabled || tt || n == 0) return PERFT_OK;
    int d = 0;
    for (u32 i = 0; i < n; i++) d = std::max<int>(d, depths[i]);
    if (d > DD_MAX_LEVELS) return PERFT_OK;
    // the graph path has the two Kogge-Stone instantiations; another tuned
    // variant runs there as plain Kogge-Stone (same counts)
    auto ddSv = [](int v) { return (v == SV_KOGGE || v == SV_KOGGE_SPLIT) ? v : (int)SV_KOGGE; };
    const int ddL = ddSv(svLeaf), ddE = ddSv(svExpand);
    DDGraph *G = nullptr;
    for (DDGraph &g : ddCache)
        if (g.depth == d && g.n == n && g.dPos == dPos && g.dOut == dOut && g.top == arenaTop && g.svL == ddL &&
            g.svE == ddE && memcmp(g.depths.data(), depths, n) == 0)
            G = &g;
    if (G && G->overflowed) return PERFT_OK;
    std::vector<double> predLv;
    if (!G && !ddForce) {
        // Predicted bytes of the materialised plies: each root's own move
        // count times 32 per further ply (the measured mean is about 30),
        // 72 bytes per node.  The positions are read back once, when the
        // graph is built; a replay needs no prediction.
        std::vector<u64> hp(6ull * n);
        ENG_TRY(cudaMemcpyAsync(hp.data(), dPos, 48ull * n, cudaMemcpyDeviceToHost, stream));
        ENG_TRY(cudaStreamSynchronize(stream));
        double est = 0;
        predLv.assign(DD_MAX_LEVELS, 0.0);
        for (u32 i = 0; i < n; i++) {
            if (depths[i] < 2 || validate_pos48(&hp[6ull * i]) != 0) continue;
            const int join = d - depths[i];  // the level this root enters
            predLv[join] += 1.0;
            double nodes = (double)count_moves<SV_KOGGE>(from_pos48(&hp[6ull * i])), sum = 0;
            for (int k = 1; k <= (int)depths[i] - 2; k++) {
                sum += nodes;
                predLv[join + k] += nodes;
                nodes *= 32.0;
            }
            est += sum * 72.0;
        }
        if (est > 0.85 * (double)arena_free()) return PERFT_OK;
        if (est > ddMaxBytes) return PERFT_OK;
    }
    if (!G) {
        if (ddCache.size() >= 16) {
            DDGraph &old = ddCache.front();
            if (old.exec) cudaGraphExecDestroy(old.exec);
            if (old.graph) cudaGraphDestroy(old.graph);
            cudaFreeHost(old.hTemplate);
            cudaFreeHost(old.hIds);
            cudaFreeHost(old.hFlags);
            if (old.evLeaf0) cudaEventDestroy(old.evLeaf0);
            if (old.evLeaf1) cudaEventDestroy(old.evLeaf1);
            ddCache.erase(ddCache.begin());
        }
        ddCache.emplace_back();
        G = &ddCache.back();
        G->depth = d;
        G->depths.assign(depths, depths + n);
        G->n = n;
        G->dPos = dPos;
        G->dOut = dOut;
        G->top = arenaTop;
        G->svL = ddL;
        G->svE = ddE;
        G->predLv = predLv;
        const int rc = build_dd(*G);
        if (rc != PERFT_OK) {
            drop_dd();
            return rc == PERFT_ERR_OUT_OF_MEMORY ? PERFT_OK : rc;
        }
    }
    G->hFlags[2] = G->hFlags[3] = 0;
    ENG_TRY(cudaGraphLaunch(G->exec, stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    stats.other_launches += G->otherLaunches;
    stats.expand_launches += d > 2 ? d - 2 : 0;
    stats.leaf_launches += d >= 2 ? 1 : 0;
    stats.graph_launches += 1;
    if ((u32)G->hFlags[0]) {  // overflow: rerun host-driven, now and on later calls
        G->overflowed = true;
        return PERFT_OK;
    }
    const u32 e = (u32)G->hFlags[1];
    if (e & DERR_BAD_POSITION) return PERFT_ERR_INVALID_ARG;
    if (e) return PERFT_ERR_INTERNAL;
    stats.leaf_items += G->hFlags[2];
    stats.leaf_parents += G->hFlags[3];
    if (d >= 2) {
        float ms = 0.f;  // the count-only ply's device time, from the events recorded in the graph
        if (cudaEventElapsedTime(&ms, G->evLeaf0, G->evLeaf1) == cudaSuccess) stats.leaf_ms += ms;
        else cudaGetLastError();  // a statistic only: leave no error behind for the caller
    }
    handled = true;
    return PERFT_OK;
}

// One position of depth 2..5: the whole tree in one k_small_tree launch and
// one 16-byte read-back (count and flags).  Not handled (the level pipeline
// runs it) when disabled, outside those depths, or when the position has more
// depth-5 subtree roots than a CTA can list.  With hOut the count is also
// returned to the host from the same read-back.
int Engine::run_small(const u64 *dPos, int depth, u64 *dOut, u64 *hOut, bool &handled)
{
    handled = false;
    if (!smallEnabled || depth < 2 || depth > SMALL_MAX_DEPTH) return PERFT_OK;
    k_small_tree<SV_KOGGE><<<smallGrid, SMALL_NT, SMALL_DYN_SMEM, stream>>>(dPos, depth, smallListCap, dOut,
                                                                            dSmall);
    ENG_TRY(cudaGetLastError());
    ENG_TRY(cudaMemcpyAsync(hPinned + 4, &dSmall->count, 16, cudaMemcpyDeviceToHost, stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    const u32 flags = (u32)hPinned[5];
    if (flags & DERR_BAD_POSITION) return PERFT_ERR_INVALID_ARG;
    if (flags) return PERFT_OK;  // too many subtree roots for one CTA's list
    if (hOut) *hOut = hPinned[4];
    stats.small_launches += 1;
    handled = true;
    return PERFT_OK;
}

int Engine::run_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out)
{
    ENG_TRY(cudaSetDevice(device));  // the staging buffers and the stream belong to the engine's device
    if (n > ioCap) {
        if (ioPos) cudaFree(ioPos);
        if (ioOut) cudaFree(ioOut);
        ioPos = ioOut = nullptr;
        ioCap = 0;
        u32 cap = 1024;
        while (cap < n) cap *= 2;
        ENG_TRY(cudaMalloc(&ioPos, 48ull * cap));
        ENG_TRY(cudaMalloc(&ioOut, 8ull * cap));
        ioCap = cap;
        drop_dd();
    }
    ENG_TRY(cudaMemcpyAsync(ioPos, pos, 48ull * n, cudaMemcpyHostToDevice, stream));
    if (n == 1) {
        bool handled = false;
        const int rc = run_small(ioPos, depths[0], ioOut, out, handled);
        if (rc != PERFT_OK || handled) return rc;
    }
    const int rc = run_batch(ioPos, depths, n, ioOut, false);
    if (rc != PERFT_OK) return rc;
    ENG_TRY(cudaMemcpyAsync(out, ioOut, 8ull * n, cudaMemcpyDeviceToHost, stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    return PERFT_OK;
}

int Engine::sync_and_check_errors()
{
    ENG_TRY(cudaMemcpyAsync(hPinned + 1, dErr, 4, cudaMemcpyDeviceToHost, stream));
    ENG_TRY(cudaStreamSynchronize(stream));
    const u32 e = (u32)hPinned[1];
    if (e & DERR_BAD_POSITION) return PERFT_ERR_INVALID_ARG;
    if (e) return PERFT_ERR_INTERNAL;
    return PERFT_OK;
}

int Engine::run_batch(const u64 *dPos, const uint8_t *depths, u32 n, u64 *dOut, bool trySmall)
{
    ENG_TRY(cudaSetDevice(device));
    if (n == 1 && trySmall) {
        bool handled = false;
        const int rc = run_small(dPos, depths[0], dOut, nullptr, handled);
        if (rc != PERFT_OK || handled) return rc;
    }
    {
        bool handled = false;
        const int rc = run_dd(dPos, depths, n, dOut, handled);
        if (rc != PERFT_OK || handled) return rc;
    }
    const u64 mark0 = arenaTop;
    unsigned long long *rootCounts = (unsigned long long *)dOut;
    ENG_TRY(cudaMemsetAsync(rootCounts, 0, 8ull * n, stream));
    ENG_TRY(cudaMemsetAsync(dErr, 0, 4, stream));

    // group roots by depth: every node of a level then has the same remaining depth
    std::map<int, std::vector<u32>, std::greater<int>> groups;
    for (u32 i = 0; i < n; i++) groups[depths[i]].push_back(i);

    int rc = PERFT_OK;
    if (!tt) {
        // Without a table all depth groups share their plies: the deepest
        // roots start, the others join the level of their remaining depth,
        // so the batch takes one launch per ply (chunked only where a level
        // does not fit the arena).  Roots of depth 0 and 1 are answered by
        // k_init_roots alone.
        std::vector<u32> order;
        order.reserve(n);
        Joiners J;
        J.dPos = dPos;
        std::vector<std::pair<int, size_t>> offs;
        for (auto &g : groups) {
            offs.push_back({g.first, order.size()});
            order.insert(order.end(), g.second.begin(), g.second.end());
        }
        u32 *dIds = (u32 *)alloc(4ull * n);
        if (!dIds) rc = PERFT_ERR_OUT_OF_MEMORY;
        if (rc == PERFT_OK) {
            ENG_TRY(cudaMemcpyAsync(dIds, order.data(), 4ull * n, cudaMemcpyHostToDevice, stream));
            for (auto &o : offs) {
                J.ids[o.first] = dIds + o.second;
                J.n[o.first] = (u32)groups[o.first].size();
            }
            const int dmax = groups.begin()->first;
            // the shallow roots (depth 0, 1) in one scratch level each
            for (int d = 0; d <= 1 && rc == PERFT_OK; d++) {
                if (!J.n[d]) continue;
                const u64 gm = arenaTop;
                DeviceLevel S;
                if (!alloc_level(S, J.n[d])) rc = PERFT_ERR_OUT_OF_MEMORY;
                else rc = init_joiners(J, d, S, 0, rootCounts);
                arenaTop = gm;
            }
            if (rc == PERFT_OK && dmax >= 2) {
                DeviceLevel L0;
                if (!alloc_level(L0, J.n[dmax])) rc = PERFT_ERR_OUT_OF_MEMORY;
                if (rc == PERFT_OK) rc = init_joiners(J, dmax, L0, 0, rootCounts);
                if (rc == PERFT_OK) rc = sync_and_check_errors();
                if (rc == PERFT_OK) rc = process_level(L0, dmax, rootCounts, &J);
            }
        }
        groups.clear();  // done: skip the per-group loop below
    }
    for (auto &g : groups) {
        const int depth = g.first;
        const std::vector<u32> &ids = g.second;
        const u64 gm = arenaTop;
        u32 *dIds = (u32 *)alloc(4ull * ids.size());
        DeviceLevel L0;
        if (!dIds || !(tt ? alloc_level_tt(L0, ids.size()) : alloc_level(L0, ids.size()))) {
            rc = PERFT_ERR_OUT_OF_MEMORY;
            break;
        }
        ENG_TRY(cudaMemcpyAsync(dIds, ids.data(), 4ull * ids.size(), cudaMemcpyHostToDevice, stream));
        const u32 nb = (u32)((ids.size() + 127) / 128);
        k_init_roots<<<nb, 128, 0, stream>>>(dPos, dIds, (u32)ids.size(), L0.planes, L0.stride, L0.cnt,
                                              L0.root, depth, rootCounts, dErr);
        stats.other_launches++;
        ENG_TRY(cudaGetLastError());
        rc = sync_and_check_errors();
        if (rc != PERFT_OK) break;
        if (depth >= 2) rc = tt ? process_level_tt(L0, depth, nullptr, rootCounts) : process_level(L0, depth, rootCounts);
        arenaTop = gm;
        if (rc != PERFT_OK) break;
    }
    arenaTop = mark0;
    if (rc != PERFT_OK) {
        cudaStreamSynchronize(stream);
        return rc;
    }
    rc = sync_and_check_errors();
    stats.peak_arena_bytes = std::max<u64>(stats.peak_arena_bytes, arenaPeak);
    return rc;
}

// ================================================================ C ABI glue
Engine g_engine;

}  // namespace

#include "serve.cuh"

namespace pg {
// Shared with host.cpp: run a batch on the process-wide engine (host buffers).
int engine_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out);
}

int pg::engine_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out)
{
    Engine &E = g_engine;
    std::lock_guard<std::mutex> lk(E.mu);
    if (!E.ready) return PERFT_ERR_NOT_INITIALIZED;
    if (n == 0) return PERFT_OK;
    for (u32 i = 0; i < n; i++) {
        if (validate_pos48(pos + 6ull * i) != 0) return PERFT_ERR_INVALID_ARG;
        if (depths[i] > 20) return PERFT_ERR_INVALID_ARG;
    }
    return E.run_batch_host(pos, depths, n, out);
}

extern "C" {

void perft_config_default(perft_config *cfg)
{
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->device = 0;
    cfg->arena_bytes = 0;
    cfg->sliders_expand = PERFT_SLIDERS_AUTO;
    cfg->sliders_leaf = PERFT_SLIDERS_AUTO;
    cfg->tt_log2_entries = 0;
    cfg->zobrist_seed = 0x5EED0781ULL;
}

int perft_init(const perft_config *cfg)
{
    perft_config c;
    if (cfg) c = *cfg;
    else perft_config_default(&c);
    if (g_server.running) perft_serve_stop();
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (g_engine.ready) g_engine.shutdown();
    return g_engine.init(c);
}

int perft_shutdown(void)
{
    if (g_server.running) perft_serve_stop();
    std::lock_guard<std::mutex> lk(g_engine.mu);
    g_engine.shutdown();
    return PERFT_OK;
}

void perft_serve_config_default(perft_serve_config *cfg)
{
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->memory_bytes = 0;
    cfg->step_items = 1ull << 27;
    cfg->max_in_flight = 4096;
    cfg->use_tt = 1;
}

int perft_serve_start(const perft_serve_config *cfg)
{
    perft_serve_config c;
    if (cfg) c = *cfg;
    else perft_serve_config_default(&c);
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (!g_engine.ready) return PERFT_ERR_NOT_INITIALIZED;
    if (g_server.running) return PERFT_ERR_INVALID_ARG;
    const u64 fixed = 256ull << 20;  // slot tables, staging, scratch
    u64 bytes = c.memory_bytes ? c.memory_bytes + fixed : (u64)(g_engine.free_bytes() * 0.9);
    if (bytes > g_engine.free_bytes()) return PERFT_ERR_OUT_OF_MEMORY;
    char *block = g_engine.reserve_block(bytes);
    if (!block) return PERFT_ERR_OUT_OF_MEMORY;
    const int rc = g_server.start(c, block, bytes, g_engine.device_id());
    if (rc != PERFT_OK) g_engine.release_block();
    return rc;
}

int perft_serve_stop(void)
{
    const bool was = g_server.running;
    const int rc = g_server.stop();
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (was && g_engine.ready) g_engine.release_block();
    return rc;
}

int perft_serve_submit(const perft_pos48 *pos, uint32_t depth, uint64_t *ticket)
{
    if (!pos || !ticket) return PERFT_ERR_INVALID_ARG;
    if (!g_server.running) return PERFT_ERR_NOT_INITIALIZED;
    return g_server.submit(pos->bb, depth, ticket);
}

int perft_serve_poll(uint64_t ticket, uint64_t *count, double *latency_s)
{
    return g_server.poll(ticket, count, latency_s, false, 0.0);
}

int perft_serve_wait(uint64_t ticket, double timeout_s, uint64_t *count, double *latency_s)
{
    return g_server.poll(ticket, count, latency_s, true, timeout_s);
}

int perft_serve_get_stats(perft_serve_stats *out)
{
    if (!out) return PERFT_ERR_INVALID_ARG;
    memset(out, 0, sizeof *out);
    g_server.get_stats(out);
    return PERFT_OK;
}

const char *perft_status_string(int status)
{
    switch (status) {
    case PERFT_OK: return "ok";
    case PERFT_ERR_INVALID_ARG: return "invalid argument";
    case PERFT_ERR_NOT_INITIALIZED: return "engine not initialized (call perft_init)";
    case PERFT_ERR_CUDA: return "CUDA error";
    case PERFT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case PERFT_ERR_INTERNAL: return "internal consistency check failed on the device";
    case PERFT_ERR_BAD_FEN: return "malformed FEN";
    case PERFT_ERR_NO_DEVICE: return "no CUDA device";
    case PERFT_ERR_ILLEGAL_MOVE: return "illegal move";
    case PERFT_ERR_TIMEOUT: return "timed out";
    case PERFT_ERR_NOT_FOUND: return "not found";
    case PERFT_ERR_IO: return "file I/O error";
    case PERFT_ERR_OVERFLOW: return "count does not fit 64 bits";
    default: return "unknown status";
    }
}

int perft(const perft_pos48 *pos, uint32_t depth, uint64_t *out)
{
    if (!pos || !out || depth > 255) return PERFT_ERR_INVALID_ARG;
    uint8_t d = (uint8_t)depth;
    return pg::engine_batch_host(pos->bb, &d, 1, out);
}

int perft_batch(const perft_pos48 *pos, const uint8_t *depths, uint32_t n, uint64_t *out)
{
    if ((!pos || !depths || !out) && n) return PERFT_ERR_INVALID_ARG;
    return pg::engine_batch_host(pos ? pos->bb : nullptr, depths, n, out);
}

int perft_batch_device(const perft_pos48 *d_pos, const uint8_t *depths, uint32_t n, uint64_t *d_out)
{
    if ((!d_pos || !depths || !d_out) && n) return PERFT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (!g_engine.ready) return PERFT_ERR_NOT_INITIALIZED;
    for (u32 i = 0; i < n; i++)
        if (depths[i] > 20) return PERFT_ERR_INVALID_ARG;
    if (n == 0) return PERFT_OK;
    return g_engine.run_batch(d_pos->bb, depths, n, d_out);
}

int perft_get_stats(perft_stats *out)
{
    if (!out) return PERFT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (g_engine.ready) g_engine.read_tt_stats();
    *out = g_engine.stats;
    return PERFT_OK;
}

int perft_get_tuning(perft_tune_entry *out, uint32_t cap, uint32_t *n)
{
    if (!n || (!out && cap)) return PERFT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (!g_engine.ready) return PERFT_ERR_NOT_INITIALIZED;
    uint32_t k = 0;
    auto put = [&](int leaf, int r) {
        const Engine::TuneCfg &c = g_engine.tuneTab[leaf ? MODE_LEAF : MODE_EXPAND][r];
        if (k < cap) out[k] = perft_tune_entry{leaf, r, c.sv, c.cap, c.ctas, c.ms};
        k++;
    };
    put(1, 2);
    for (int r = 3; r <= g_engine.tunedMaxR; r++) put(0, r);
    *n = k;
    return k <= cap ? PERFT_OK : PERFT_ERR_INVALID_ARG;
}

int perft_tt_clear(void)
{
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (!g_engine.ready) return PERFT_ERR_NOT_INITIALIZED;
    return g_engine.tt_clear();
}

int perft_reset_stats(void)
{
    std::lock_guard<std::mutex> lk(g_engine.mu);
    if (g_engine.ready) g_engine.zero_tt_stats();
    perft_stats keep = g_engine.stats;
    memset(&g_engine.stats, 0, sizeof g_engine.stats);
    g_engine.stats.sliders_expand = keep.sliders_expand;
    g_engine.stats.sliders_leaf = keep.sliders_leaf;
    g_engine.stats.arena_bytes = keep.arena_bytes;
    return PERFT_OK;
}

}  // extern "C"

// ======================================================= allocation-free entry
// perft_batch_noalloc: the batched perft for callers that cannot allocate
// device memory — processes whose HBM is already reserved by another
// allocator (a serving framework or torch's caching allocator holding the
// device), and latency-critical callers for which cudaMalloc's implicit
// device-wide synchronisation is unacceptable.  It runs the same kernels as
// perft_batch_device, but every level buffer, scan, tile index and counter
// lives in one fixed scratch array compiled into this library, so the call
// allocates nothing.  Trees whose levels do not fit the scratch are refused
// (PERFT_ERR_OUT_OF_MEMORY); the arena engine handles those by chunking.
//
// The scratch is a file-scope __device__ array: every GPU that loads this
// library holds NOALLOC_SCRATCH_BYTES of it until the process exits.  All
// calls on a device share it and it keeps the previous call's contents, so
// each call clears its counters and outputs first.  Two calls whose GPU work
// overlapped would corrupt each other: this entry point takes a process-wide
// lock and waits for its stream before returning, on error paths too, so its
// own calls never overlap.  The first call on a device uploads the
// move-generator tables and looks up the scratch address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture.
static __device__ __align__(256) unsigned char g_noallocScratch[PERFT_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;

struct NoallocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noallocScratch
    int gridLeaf = 0, gridExpand = 0;
};

std::mutex g_noallocMu;
NoallocDevice g_noallocDev[NOALLOC_MAX_DEVICES];

// Writes, in order, the indices of the roots whose depth equals `depth`.
__global__ void __launch_bounds__(1024) k_noalloc_group_ids(const uint8_t *__restrict__ depths, u32 n,
                                                            int depth, u32 *__restrict__ ids,
                                                            u32 *__restrict__ count)
{
    __shared__ int sw[32];
    u32 base = 0;
    for (u32 c0 = 0; c0 < n; c0 += 1024) {
        const u32 i = c0 + threadIdx.x;
        const bool hit = i < n && depths[i] == depth;
        int tot = 0;
        const int r = block_excl_count<1024>(hit, sw, tot);
        if (hit) ids[base + r] = i;
        base += (u32)tot;
    }
    if (threadIdx.x == 0) *count = base;
}

// Looks up the scratch address with `dev` current, on every call: the lookup
// allocates nothing and is cheap.  If the address differs from the one cached
// (first call on the device, or the device's primary context was destroyed and
// created again, e.g. by cudaDeviceReset), the move tables are uploaded into
// the current context before the address is trusted.
int noalloc_setup(int dev)
{
    NoallocDevice &D = g_noallocDev[dev];
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noallocScratch) != cudaSuccess || p == nullptr) return PERFT_ERR_CUDA;
    if (D.ready && D.scratch == (unsigned char *)p) return PERFT_OK;
    D.ready = false;
    build_tables();
    if (cudaMemcpyToSymbol(d_tables, &h_tables, sizeof(Tables)) != cudaSuccess) return PERFT_ERR_CUDA;
    if (cudaMemcpyToSymbol(d_magic, h_magic, sizeof(h_magic)) != cudaSuccess) return PERFT_ERR_CUDA;
    u32 pow2[32];
    for (int k = 0; k < 32; k++) pow2[k] = 1u << k;
    if (cudaMemcpyToSymbol(c_pow2, pow2, sizeof pow2) != cudaSuccess) return PERFT_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return PERFT_ERR_CUDA;
    D.scratch = (unsigned char *)p;
    D.gridLeaf = occupancy_grid<MODE_LEAF, SV_KOGGE>(prop.multiProcessorCount);
    D.gridExpand = occupancy_grid<MODE_EXPAND, SV_KOGGE>(prop.multiProcessorCount);
    D.ready = true;
    return PERFT_OK;
}

// One call's bump allocator over the static scratch, and the level loop
// without chunking.
struct NoallocRun {
    unsigned char *base;
    u64 top = 0;
    cudaStream_t st;
    u32 *counter = nullptr, *err = nullptr;
    int gridLeaf = 0, gridExpand = 0;

    void *take(u64 bytes)
    {
        const u64 a = (top + 255) & ~255ULL;
        if (a + bytes > PERFT_NOALLOC_SCRATCH_BYTES) return nullptr;
        top = a + bytes;
        return base + a;
    }

    bool level(DeviceLevel &L, u64 n)
    {
        L.n = n;
        L.stride = (n + 31) & ~31ULL;
        L.planes = (u64 *)take(6 * 8 * L.stride);
        L.cnt = (u32 *)take(4 * L.stride);
        L.root = (u32 *)take(4 * L.stride);
        return L.planes && L.cnt && L.root;
    }

    int read_u64(const u64 *src, u64 &v)
    {
        if (cudaMemcpyAsync(&v, src, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PERFT_ERR_CUDA;
        return cudaStreamSynchronize(st) == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
    }

    int scan(const u32 *cnt, u64 n, u64 *&scanOut, u32 *&tileFirst, u64 &total)
    {
        const u64 nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
        const u64 maxTiles = (n * MAX_LEGAL_MOVES + TILE_CAP - 1) / TILE_CAP + 1;
        scanOut = (u64 *)take(8 * (n + 1));
        tileFirst = (u32 *)take(4 * maxTiles);
        u64 *bsum = (u64 *)take(8 * (nb + 1));
        if (!scanOut || !tileFirst || !bsum) return PERFT_ERR_OUT_OF_MEMORY;
        k_scan_reduce<<<(unsigned)nb, SCAN_NT, 0, st>>>(cnt, n, bsum);
        k_scan_top<<<1, SCAN_TOP_NT, 0, st>>>(bsum, nb, scanOut + n);
        k_scan_apply<<<(unsigned)nb, SCAN_NT, 0, st>>>(cnt, n, bsum, scanOut, tileFirst, TILE_CAP_LOG2);
        if (cudaGetLastError() != cudaSuccess) return PERFT_ERR_CUDA;
        return read_u64(scanOut + n, total);
    }

    int tile(int mode, const DeviceLevel &par, const u64 *pscan, const u32 *tileFirst, u64 total,
             DeviceLevel *ch, unsigned long long *rootCounts)
    {
        TileParams P;
        memset(&P, 0, sizeof P);
        P.ppl = par.planes;
        P.pstride = par.stride;
        P.pscan = pscan;
        P.proot = par.root;
        P.nParents = par.n;
        P.tileFirst = tileFirst;
        P.itemBase = 0;
        P.itemEnd = total;
        P.capLog2 = TILE_CAP_LOG2;
        P.tileCounter = counter;
        if (ch) {
            P.cpl = ch->planes;
            P.cstride = ch->stride;
            P.ccnt = ch->cnt;
            P.croot = ch->root;
        }
        P.rootCounts = rootCounts;
        P.err = err;
        const u64 nTiles = (total + TILE_CAP - 1) / TILE_CAP;
        if (cudaMemsetAsync(counter, 0, 4, st) != cudaSuccess) return PERFT_ERR_CUDA;
        if (mode == MODE_LEAF)
            launch_tile_variant<MODE_LEAF>(SV_KOGGE, (int)std::min<u64>(gridLeaf, nTiles), st, P);
        else
            launch_tile_variant<MODE_EXPAND>(SV_KOGGE, (int)std::min<u64>(gridExpand, nTiles), st, P);
        return cudaGetLastError() == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
    }

    int process(const DeviceLevel &L, int remaining, unsigned long long *rootCounts)
    {
        if (L.n == 0) return PERFT_OK;
        u64 *pscan = nullptr;
        u32 *tileFirst = nullptr;
        u64 total = 0;
        int rc = scan(L.cnt, L.n, pscan, tileFirst, total);
        if (rc != PERFT_OK || total == 0) return rc;
        if (remaining == 2) return tile(MODE_LEAF, L, pscan, tileFirst, total, nullptr, rootCounts);
        const u64 mark = top;
        DeviceLevel C;
        if (!level(C, total)) return PERFT_ERR_OUT_OF_MEMORY;
        rc = tile(MODE_EXPAND, L, pscan, tileFirst, total, &C, nullptr);
        if (rc == PERFT_OK) rc = process(C, remaining - 1, rootCounts);
        top = mark;
        return rc;
    }
};

}  // namespace

extern "C" int perft_batch_noalloc(const perft_pos48 *d_pos, const uint8_t *depths, uint32_t n,
                                   uint64_t *d_out, void *stream)
{
    if ((!d_pos || !depths || !d_out) && n) return PERFT_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++)
        if (depths[i] > 20) return PERFT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_noallocMu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PERFT_ERR_NO_DEVICE;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PERFT_ERR_INVALID_ARG;
    int rc = noalloc_setup(dev);
    if (rc != PERFT_OK || n == 0) return rc;

    NoallocRun R;
    R.base = g_noallocDev[dev].scratch;
    R.st = (cudaStream_t)stream;
    R.gridLeaf = g_noallocDev[dev].gridLeaf;
    R.gridExpand = g_noallocDev[dev].gridExpand;
    R.counter = (u32 *)R.take(4);
    R.err = (u32 *)R.take(4);
    u32 *dIds = (u32 *)R.take(4ull * n);
    uint8_t *dDepths = (uint8_t *)R.take(n);
    u32 *dGroupCount = (u32 *)R.take(4);
    if (!R.counter || !R.err || !dIds || !dDepths || !dGroupCount) return PERFT_ERR_OUT_OF_MEMORY;

    // From the first queued operation on, every return goes through the
    // stream synchronisation at the end, so the call never returns with work
    // of its own still queued on the shared scratch (a failed call included).
    unsigned long long *rootCounts = (unsigned long long *)d_out;
    if (cudaMemsetAsync(R.err, 0, 4, R.st) != cudaSuccess ||
        cudaMemsetAsync(rootCounts, 0, 8ull * n, R.st) != cudaSuccess ||
        cudaMemcpyAsync(dDepths, depths, n, cudaMemcpyHostToDevice, R.st) != cudaSuccess)
        rc = PERFT_ERR_CUDA;

    // Group roots by depth without host allocation: the depths go to the
    // scratch and a kernel compacts the ids of one depth group in order.
    u32 perDepth[21] = {0};
    for (u32 i = 0; i < n; i++) perDepth[depths[i]]++;
    for (int depth = 20; depth >= 0 && rc == PERFT_OK; depth--) {
        const u32 cnt = perDepth[depth];
        if (!cnt) continue;
        const u64 mark = R.top;
        DeviceLevel L0;
        if (!R.level(L0, cnt)) {
            rc = PERFT_ERR_OUT_OF_MEMORY;
            break;
        }
        k_noalloc_group_ids<<<1, 1024, 0, R.st>>>(dDepths, n, depth, dIds, dGroupCount);
        k_init_roots<<<(cnt + 127) / 128, 128, 0, R.st>>>(d_pos->bb, dIds, cnt, L0.planes, L0.stride,
                                                           L0.cnt, L0.root, depth, rootCounts, R.err);
        if (cudaGetLastError() != cudaSuccess) {
            rc = PERFT_ERR_CUDA;
            break;
        }
        if (depth >= 2) rc = R.process(L0, depth, rootCounts);
        R.top = mark;
    }
    u32 e = 0;
    const bool readOk = cudaMemcpyAsync(&e, R.err, 4, cudaMemcpyDeviceToHost, R.st) == cudaSuccess;
    const bool syncOk = cudaStreamSynchronize(R.st) == cudaSuccess;
    if (rc != PERFT_OK) return rc;
    if (!readOk || !syncOk) return PERFT_ERR_CUDA;
    if (e & DERR_BAD_POSITION) return PERFT_ERR_INVALID_ARG;
    return e ? PERFT_ERR_INTERNAL : PERFT_OK;
}
