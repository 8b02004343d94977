// Continuous-batching perft server (included by engine.cu: it drives the
// same kernels).
//
// Queries of mixed depth arrive at any time.  Each admitted query owns a
// slot; its frontier lives in HBM as level buffers, kept in pools by
// remaining depth, and the levels of different queries with the same
// remaining depth are advanced by the same kernels.  One scheduler iteration:
//   1. admit queued queries while slots are free and the predicted
//      level-buffer memory of all admitted queries fits the budget;
//   2. advance every pool, the count-only last ply first, each level by at
//      most `step_items` (tile-aligned), so a large level never blocks the
//      small levels of newer queries for more than one step;
//   3. read back the per-query pending-node counters (maintained on the
//      device by the tracking tile kernels) and complete every query whose
//      counter reached zero.
// Work of different queries therefore overlaps on the device, queries that
// arrive while others run join at the next iteration, and no query waits for
// another to finish.  A query's count is the same alone or in the mix: it
// is a sum of exact per-item counts, only the grouping into launches varies.
//
// Transposition table: with an engine table and use_tt, every level two or
// three plies above the leaves (remaining depth 2 or 3) is hashed and probed
// before its scan, exactly as the engine's own table levels are (k_tt_probe,
// k_tt_dedup): table hits take the stored count and generate nothing, and
// identical nodes of the level are searched once.  Counts then flow up per
// node, not per query:
//   * a remaining-depth-3 level expands without pending-count tracking; each
//     child level (remaining depth 2) it produces sums its leaf ply per node
//     and, when done, stores its nodes and adds each node's count into its
//     parent's sum (the engine's k_tt_finish);
//   * once a remaining-depth-3 level is fully expanded and all its child
//     levels are done, it is finished like a remaining-depth-2 level of a
//     depth-2 query: its searched nodes are stored, duplicates take their
//     owner's count, and every node's count goes to its query, whose pending
//     count drops by one per node (k_serve_tt_finish).
// The table lives in the engine for the life of the process, so it is shared
// by all queries and keeps its entries across queries.
#pragma once

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

constexpr u32 SERVE_MAX_SLOTS = 1u << 16;
constexpr int SERVE_MAX_R = 21;

__global__ void k_serve_admit(const u64 *__restrict__ stagePos, const u32 *__restrict__ slots,
                              const uint8_t *__restrict__ depths, u32 n, u64 *__restrict__ posBySlot,
                              unsigned long long *__restrict__ pending, unsigned long long *__restrict__ counts)
{
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 s = slots[i];
#pragma unroll
    for (int k = 0; k < 6; k++) posBySlot[6ull * s + k] = stagePos[6ull * i + k];
    counts[s] = 0;
    pending[s] = depths[i] >= 2 ? 1ull : 0ull;
}

// Parents with no legal move end their branch at scan time.
__global__ void k_serve_zero_parents(const u32 *__restrict__ cnt, const u32 *__restrict__ root, u64 n,
                                     unsigned long long *pending)
{
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && cnt[i] == 0) atomicAdd(&pending[root[i]], ~0ull);  // -1
}

struct ServeQuery {
    u64 ticket = 0;
    u64 pos[6];
    u32 depth = 0;
    int slot = -1;
    int state = 0;  // 0 queued, 1 running, 2 done
    double tSubmit = 0, tAdmit = 0, tDone = 0;
    u64 predicted = 0;
    u64 result = 0;
};

// Last step of a table level: owners (and nodes not de-duplicated) store
// their subtree count, duplicates take their owner's, and every node's count
// goes to its query with the node's pending mark removed (warp-aggregated per
// run of equal query slot: the nodes of a level are ordered by query).
__global__ void __launch_bounds__(256) k_serve_tt_finish(u64 n, const u64 *__restrict__ hash,
                                                         const u64 *__restrict__ hash2,
                                                         const unsigned long long *__restrict__ acc,
                                                         const u32 *__restrict__ alias, const u32 *__restrict__ slot,
                                                         unsigned long long *counts, unsigned long long *pending,
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
            v = acc[a];  // the owner's subtree finished with this level's last launch
        } else if (a != ALIAS_HIT) {
            tt[hash[i] & ttMask] = make_ulonglong2(hash2[i] ^ v, v);
            stored = true;
        }
        key = slot[i];
    }
    count_stat(&ts->stores, stored);
    // a count three plies deep is below 218^3 < 2^24, so 32 of them sum in 32 bits
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const unsigned long long sum = __reduce_add_sync(peers, (unsigned)v);
    if (i < n && lane == __ffs(peers) - 1) {
        atomicAdd(&counts[key], sum);
        atomicAdd(&pending[key], (unsigned long long)(-(long long)__popc(peers)));
    }
}

struct ServeLevel {
    DeviceLevel L;
    int r = 0;
    bool scanned = false;
    bool tt = false;  // a table level: per-node sums, finished by k_serve_tt_finish
    // a remaining-depth-2 level expanded from a table level of remaining depth
    // 3: its root array holds parent indices into that level, its counts go
    // into the parent's sums (k_tt_finish)
    struct ServeLevel *parent = nullptr;
    int outstanding = 0;  // (table levels of remaining depth 3) child levels not yet finished
    std::vector<std::pair<u64, u64>> ttMem;  // its hashes, sums and aliases
    u64 *pscan = nullptr;
    u32 *tileFirst = nullptr;
    u64 total = 0, next = 0;
    std::vector<std::pair<u64, u64>> mem;  // (offset, bytes) in the server block
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

class Server {
public:
    int start(const perft_serve_config &cfg, char *block, u64 bytes, int device);
    int stop();
    int submit(const u64 pos[6], u32 depth, u64 *ticket);
    int poll(u64 ticket, u64 *count, double *latency, bool wait, double timeoutS);
    void get_stats(perft_serve_stats *out);
    bool running = false;
    char *blockBase = nullptr;

private:
    // ---- device-memory first-fit allocator over the server's arena block
    u64 blockBytes = 0;
    std::map<u64, u64> freeRanges;  // offset -> size
    u64 inUse = 0, peakInUse = 0;
    void *take(u64 bytes, std::vector<std::pair<u64, u64>> &owner);
    void give_back(std::vector<std::pair<u64, u64>> &owner);

    void loop();
    int admit();
    int advance();
    int complete();
    int scan_level(ServeLevel &S);
    int launch(int mode, ServeLevel &S, u64 lo, u64 hi, DeviceLevel *child);
    int probe_level(ServeLevel &S);
    int finish_level(ServeLevel &S);
    int retire(ServeLevel *S);
    std::vector<ServeLevel *> waiting;  // table levels fully expanded, waiting for their child levels

    std::thread worker;
    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    bool stopping = false;
    std::deque<ServeQuery *> queue;
    std::unordered_map<u64, ServeQuery *> byTicket;
    std::vector<ServeQuery *> bySlot;
    std::vector<u32> freeSlots;
    u64 nextTicket = 1;

    int dev = 0;
    cudaStream_t st = nullptr;
    u32 *dErr = nullptr, *dCounter = nullptr;
    u64 *posBySlot = nullptr;
    unsigned long long *pending = nullptr, *counts = nullptr;
    u64 *hostPending = nullptr, *hostCounts = nullptr, *hostTotal = nullptr;  // pinned
    u64 *stagePos = nullptr;   // pinned
    u32 *stageSlots = nullptr; // pinned
    uint8_t *stageDepths = nullptr;
    std::vector<std::pair<u64, u64>> fixedMem;
    std::vector<ServeLevel *> pools[SERVE_MAX_R + 1];
    u64 budget = 0, reserved = 0, stepItems = 0;
    u32 maxInFlight = 0, inFlight = 0, maxSlotUsed = 0;
    int gridLeaf = 0, gridExpand = 0, gridLeafAcc = 0, gridExpandTT = 0;
    bool leafSplit = false;
    // the engine's transposition table, when the server uses it
    ulonglong2 *tt = nullptr;
    u64 ttMask = 0, ttKeyMask = ~0ULL;
    TTStats *dTTStats = nullptr;
    TTStats *hostTTStats = nullptr;  // pinned
    int idleIterations = 0;
    // statistics
    u64 submitted = 0, completed = 0, iterations = 0, launches = 0, admittedBatches = 0;
    int lastError = PERFT_OK;
};

void *Server::take(u64 bytes, std::vector<std::pair<u64, u64>> &owner)
{
    bytes = (bytes + 255) & ~255ULL;
    for (auto it = freeRanges.begin(); it != freeRanges.end(); ++it) {
        if (it->second < bytes) continue;
        const u64 off = it->first, rest = it->second - bytes;
        freeRanges.erase(it);
        if (rest) freeRanges[off + bytes] = rest;
        owner.push_back({off, bytes});
        inUse += bytes;
        peakInUse = std::max(peakInUse, inUse);
        return blockBase + off;
    }
    return nullptr;
}

// Returns every range of `owner`; later launches on the same stream may
// reuse it, which stream order makes safe.
void Server::give_back(std::vector<std::pair<u64, u64>> &owner)
{
    for (auto &r : owner) {
        u64 off = r.first, size = r.second;
        inUse -= size;
        auto nx = freeRanges.lower_bound(off);
        if (nx != freeRanges.end() && off + size == nx->first) {
            size += nx->second;
            nx = freeRanges.erase(nx);
        }
        if (nx != freeRanges.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                pv->second += size;
                continue;
            }
        }
        freeRanges[off] = size;
    }
    owner.clear();
}

int Server::start(const perft_serve_config &cfg, char *block, u64 bytes, int device)
{
    dev = device;
    blockBase = block;
    blockBytes = bytes;
    freeRanges.clear();
    freeRanges[0] = bytes;
    inUse = peakInUse = 0;
    stepItems = cfg.step_items ? ((cfg.step_items + TILE_CAP - 1) & ~(u64)(TILE_CAP - 1)) : (1ull << 27);
    maxInFlight = cfg.max_in_flight ? std::min(cfg.max_in_flight, SERVE_MAX_SLOTS) : 4096;
    if (cudaSetDevice(dev) != cudaSuccess) return PERFT_ERR_CUDA;
    if (cudaStreamCreate(&st) != cudaSuccess) return PERFT_ERR_CUDA;
    posBySlot = (u64 *)take(48ull * SERVE_MAX_SLOTS, fixedMem);
    pending = (unsigned long long *)take(8ull * SERVE_MAX_SLOTS, fixedMem);
    counts = (unsigned long long *)take(8ull * SERVE_MAX_SLOTS, fixedMem);
    dCounter = (u32 *)take(256, fixedMem);
    dErr = (u32 *)take(256, fixedMem);
    dTTStats = (TTStats *)take(256, fixedMem);
    if (!posBySlot || !pending || !counts || !dCounter || !dErr || !dTTStats) return PERFT_ERR_OUT_OF_MEMORY;
    if (cudaMemsetAsync(dErr, 0, 4, st) != cudaSuccess) return PERFT_ERR_CUDA;
    if (cudaMemsetAsync(dTTStats, 0, sizeof(TTStats), st) != cudaSuccess) return PERFT_ERR_CUDA;
    {
        const Engine::TTView v = g_engine.tt_view();
        tt = cfg.use_tt ? v.table : nullptr;
        ttMask = v.mask;
        ttKeyMask = v.keyMask;
    }
    budget = std::min<u64>(cfg.memory_bytes ? cfg.memory_bytes : bytes, blockBytes - inUse);
    if (cudaMallocHost(&hostPending, 8ull * SERVE_MAX_SLOTS) != cudaSuccess ||
        cudaMallocHost(&hostCounts, 8ull * SERVE_MAX_SLOTS) != cudaSuccess ||
        cudaMallocHost(&hostTotal, 64) != cudaSuccess ||
        cudaMallocHost(&stagePos, 48ull * SERVE_MAX_SLOTS) != cudaSuccess ||
        cudaMallocHost(&stageSlots, 4ull * SERVE_MAX_SLOTS) != cudaSuccess ||
        cudaMallocHost(&stageDepths, SERVE_MAX_SLOTS) != cudaSuccess ||
        cudaMallocHost(&hostTTStats, sizeof(TTStats)) != cudaSuccess)
        return PERFT_ERR_OUT_OF_MEMORY;
    memset(hostTTStats, 0, sizeof(TTStats));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return PERFT_ERR_CUDA;
    cudaFuncSetAttribute(k_tile<MODE_LEAF, SV_KOGGE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TILE_DYN_SMEM);
    cudaFuncSetAttribute(k_tile<MODE_LEAF, SV_KOGGE_SPLIT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TILE_DYN_SMEM);
    cudaFuncSetAttribute(k_tile<MODE_EXPAND, SV_KOGGE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TILE_DYN_SMEM);
    // the count-only ply follows the engine's tuned leaf variant when it is
    // the split-shift Kogge-Stone one; every other choice uses plain Kogge-Stone
    leafSplit = g_engine.leaf_sliders() == SV_KOGGE_SPLIT;
    int perSm = 1;
    if (leafSplit)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_tile<MODE_LEAF, SV_KOGGE_SPLIT, true>, TILE_NT,
                                                      TILE_DYN_SMEM);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_tile<MODE_LEAF, SV_KOGGE, true>, TILE_NT,
                                                      TILE_DYN_SMEM);
    gridLeaf = std::max(1, perSm) * prop.multiProcessorCount;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_tile<MODE_EXPAND, SV_KOGGE, true>, TILE_NT,
                                                  TILE_DYN_SMEM);
    gridExpand = std::max(1, perSm) * prop.multiProcessorCount;
    // table levels' last ply: the engine's per-node-sum leaf kernel
    gridLeafAcc = leafSplit ? occupancy_grid<MODE_LEAF, SV_KOGGE_SPLIT>(prop.multiProcessorCount)
                            : occupancy_grid<MODE_LEAF, SV_KOGGE>(prop.multiProcessorCount);
    gridExpandTT = occupancy_grid<MODE_EXPAND, SV_KOGGE>(prop.multiProcessorCount);
    bySlot.assign(SERVE_MAX_SLOTS, nullptr);
    freeSlots.clear();
    for (u32 s = SERVE_MAX_SLOTS; s-- > 0;) freeSlots.push_back(s);
    submitted = completed = iterations = launches = admittedBatches = 0;
    reserved = 0;
    inFlight = 0;
    maxSlotUsed = 0;
    stopping = false;
    running = true;
    worker = std::thread([this] { loop(); });
    return PERFT_OK;
}

int Server::stop()
{
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!running) return PERFT_OK;
        stopping = true;
    }
    cvWork.notify_all();
    worker.join();
    cudaSetDevice(dev);
    cudaStreamSynchronize(st);
    for (int r = 0; r <= SERVE_MAX_R; r++) {
        for (ServeLevel *S : pools[r]) delete S;
        pools[r].clear();
    }
    for (ServeLevel *S : waiting) delete S;
    waiting.clear();
    for (auto &kv : byTicket) delete kv.second;
    byTicket.clear();
    queue.clear();
    cudaFreeHost(hostPending);
    cudaFreeHost(hostCounts);
    cudaFreeHost(hostTotal);
    cudaFreeHost(stagePos);
    cudaFreeHost(stageSlots);
    cudaFreeHost(stageDepths);
    cudaFreeHost(hostTTStats);
    cudaStreamDestroy(st);
    running = false;
    cvDone.notify_all();
    return PERFT_OK;
}

int Server::submit(const u64 pos[6], u32 depth, u64 *ticket)
{
    if (validate_pos48(pos) != 0 || depth > 20) return PERFT_ERR_INVALID_ARG;
    ServeQuery *q = new ServeQuery();
    memcpy(q->pos, pos, 48);
    q->depth = depth;
    q->tSubmit = now_s();
    // predicted peak frontier: root branching ^ (depth - 2) nodes of the last
    // materialised ply, 65 bytes each, with a safety margin
    const Board b = from_pos48(pos);
    double bf = std::min(45.0, std::max(20.0, (double)count_moves<SV_KOGGE>(b)));
    double nodes = 1.0;
    for (u32 k = 2; k < depth; k++) nodes *= bf;
    q->predicted = (u64)(nodes * NODE_BYTES * 1.5) + (1ull << 20);
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!running || stopping) {
            delete q;
            return PERFT_ERR_NOT_INITIALIZED;
        }
        q->ticket = nextTicket++;
        byTicket[q->ticket] = q;
        queue.push_back(q);
        submitted++;
        *ticket = q->ticket;
    }
    cvWork.notify_one();
    return PERFT_OK;
}

int Server::poll(u64 ticket, u64 *count, double *latency, bool wait, double timeoutS)
{
    std::unique_lock<std::mutex> lk(mu);
    auto it = byTicket.find(ticket);
    if (it == byTicket.end()) return PERFT_ERR_NOT_FOUND;
    ServeQuery *q = it->second;
    if (q->state != 2 && wait) {
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeoutS);
        cvDone.wait_until(lk, deadline, [&] { return q->state == 2 || !running; });
    }
    if (q->state != 2) return (wait ? PERFT_ERR_TIMEOUT : PERFT_PENDING);
    if (count) *count = q->result;
    if (latency) *latency = q->tDone - q->tSubmit;
    byTicket.erase(it);
    delete q;
    return PERFT_OK;
}

void Server::get_stats(perft_serve_stats *o)
{
    std::lock_guard<std::mutex> lk(mu);
    o->submitted = submitted;
    o->completed = completed;
    o->in_flight = inFlight;
    o->queued = queue.size();
    o->iterations = iterations;
    o->launches = launches;
    o->memory_budget = budget;
    o->memory_reserved = reserved;
    o->memory_peak = peakInUse;
    o->last_error = lastError;
    o->tt_probes = hostTTStats ? hostTTStats->probes : 0;
    o->tt_hits = hostTTStats ? hostTTStats->hits : 0;
    o->tt_merged = hostTTStats ? hostTTStats->aliases : 0;
    o->tt_stores = hostTTStats ? hostTTStats->stores : 0;
}

int Server::admit()
{
    std::vector<ServeQuery *> batch;
    {
        std::lock_guard<std::mutex> lk(mu);
        while (!queue.empty() && inFlight < maxInFlight && !freeSlots.empty()) {
            ServeQuery *q = queue.front();
            // always admit into an idle server, so one huge query cannot starve
            if (inFlight > 0 && reserved + q->predicted > budget) break;
            queue.pop_front();
            q->slot = (int)freeSlots.back();
            freeSlots.pop_back();
            q->state = 1;
            q->tAdmit = now_s();
            reserved += q->predicted;
            inFlight++;
            bySlot[q->slot] = q;
            maxSlotUsed = std::max(maxSlotUsed, (u32)q->slot + 1);
            batch.push_back(q);
        }
    }
    if (batch.empty()) return PERFT_OK;
    admittedBatches++;
    const u32 n = (u32)batch.size();
    // group by depth: every node of a level has the same remaining depth
    std::stable_sort(batch.begin(), batch.end(), [](ServeQuery *a, ServeQuery *b) { return a->depth > b->depth; });
    for (u32 i = 0; i < n; i++) {
        memcpy(stagePos + 6ull * i, batch[i]->pos, 48);
        stageSlots[i] = (u32)batch[i]->slot;
        stageDepths[i] = (uint8_t)batch[i]->depth;
    }
    std::vector<std::pair<u64, u64>> tmp;
    u64 *dPos = (u64 *)take(48ull * n, tmp);
    u32 *dSlots = (u32 *)take(4ull * n, tmp);
    uint8_t *dDepths = (uint8_t *)take(n, tmp);
    if (!dPos || !dSlots || !dDepths) {
        give_back(tmp);
        return PERFT_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemcpyAsync(dPos, stagePos, 48ull * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dSlots, stageSlots, 4ull * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dDepths, stageDepths, n, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return PERFT_ERR_CUDA;
    k_serve_admit<<<(n + 127) / 128, 128, 0, st>>>(dPos, dSlots, dDepths, n, posBySlot, pending, counts);
    launches++;
    u32 i0 = 0;
    while (i0 < n) {
        const u32 depth = batch[i0]->depth;
        u32 i1 = i0;
        while (i1 < n && batch[i1]->depth == depth) i1++;
        ServeLevel *S = new ServeLevel();
        S->r = (int)depth;
        const u64 cnt = i1 - i0;
        S->L.n = cnt;
        S->L.stride = (cnt + 31) & ~31ULL;
        S->L.planes = (u64 *)take(48 * S->L.stride, S->mem);
        S->L.cnt = (u32 *)take(4 * S->L.stride, S->mem);
        S->L.root = (u32 *)take(4 * S->L.stride, S->mem);
        if (!S->L.planes || !S->L.cnt || !S->L.root) {
            give_back(S->mem);
            delete S;
            give_back(tmp);
            return PERFT_ERR_OUT_OF_MEMORY;
        }
        k_init_roots<<<(unsigned)((cnt + 127) / 128), 128, 0, st>>>(posBySlot, dSlots + i0, (u32)cnt, S->L.planes,
                                                                     S->L.stride, S->L.cnt, S->L.root, depth,
                                                                     counts, dErr);
        launches++;
        if (depth >= 2) pools[depth].push_back(S);
        else {
            give_back(S->mem);
            delete S;
        }
        i0 = i1;
    }
    give_back(tmp);  // reused only by later launches on this stream
    return cudaGetLastError() == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
}

// Hashes and probes a level two or three plies above the leaves, and
// de-duplicates its misses; hits and duplicates get no items.  The level
// keeps the hashes, per-node sums and aliases until it is finished.
int Server::probe_level(ServeLevel &S)
{
    const u64 n = S.L.n;
    S.L.hash = (u64 *)take(8 * S.L.stride, S.ttMem);
    S.L.hash2 = (u64 *)take(8 * S.L.stride, S.ttMem);
    S.L.acc = (unsigned long long *)take(8 * S.L.stride, S.ttMem);
    S.L.alias = (u32 *)take(4 * S.L.stride, S.ttMem);
    u64 dsize = 1024;
    while (dsize < n + n / 4) dsize <<= 1;
    std::vector<std::pair<u64, u64>> tmp;
    u64 *dkey = (u64 *)take(8 * dsize, tmp);
    u32 *downer = (u32 *)take(4 * dsize, tmp);
    if (!S.L.hash || !S.L.hash2 || !S.L.acc || !S.L.alias || !dkey || !downer) {
        give_back(tmp);
        give_back(S.ttMem);  // the next iteration retries from scratch
        return PERFT_ERR_OUT_OF_MEMORY;
    }
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (cudaMemsetAsync(dkey, 0xFF, 8 * dsize, st) != cudaSuccess ||
        cudaMemsetAsync(downer, 0xFF, 4 * dsize, st) != cudaSuccess)
        return PERFT_ERR_CUDA;
    k_tt_probe<<<nb, 256, 0, st>>>(S.L.planes, S.L.stride, n, S.r, true, ttKeyMask, S.L.cnt, S.L.hash, S.L.hash2,
                                   S.L.acc, S.L.alias, tt, ttMask, dkey, downer, dsize - 1, dTTStats);
    k_tt_dedup<<<nb, 256, 0, st>>>(n, S.L.cnt, S.L.alias, downer, S.L.hash2, dTTStats);
    launches += 2;
    give_back(tmp);  // reused only by later launches on this stream
    S.tt = true;
    return cudaGetLastError() == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
}

int Server::finish_level(ServeLevel &S)
{
    const u64 n = S.L.n;
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (S.parent)  // into the parent level's per-node sums
        k_tt_finish<<<nb, 256, 0, st>>>(n, true, S.L.hash, S.L.hash2, S.L.acc, S.L.alias, S.L.root, S.parent->L.acc,
                                        tt, ttMask, dTTStats);
    else           // into the queries' counts
        k_serve_tt_finish<<<nb, 256, 0, st>>>(n, S.L.hash, S.L.hash2, S.L.acc, S.L.alias, S.L.root, counts,
                                               pending, tt, ttMask, dTTStats);
    launches++;
    return cudaGetLastError() == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
}

// A level whose items are all processed: finish it (table levels), free it,
// and finish a waiting parent whose last child level this was.  A table
// level of remaining depth 3 with child levels still running waits.
int Server::retire(ServeLevel *S)
{
    if (S->tt && S->outstanding > 0) {
        waiting.push_back(S);
        return PERFT_OK;
    }
    if (S->tt) {
        const int rc = finish_level(*S);
        if (rc != PERFT_OK) return rc;
    }
    ServeLevel *parent = S->parent;
    give_back(S->mem);
    give_back(S->ttMem);
    delete S;
    if (parent && --parent->outstanding == 0 && parent->scanned && parent->next >= parent->total) {
        auto it = std::find(waiting.begin(), waiting.end(), parent);
        if (it != waiting.end()) {
            waiting.erase(it);
            return retire(parent);
        }
    }
    return PERFT_OK;
}

int Server::scan_level(ServeLevel &S)
{
    if (tt && (S.r == 2 || S.r == 3) && !S.tt) {
        const int rc = probe_level(S);
        if (rc != PERFT_OK) return rc;
    }
    const u64 n = S.L.n;
    const u64 nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    const u64 maxTiles = (n * MAX_LEGAL_MOVES) / MAX_TILES_PER_NODE_DIV + 2;
    S.pscan = (u64 *)take(8 * (n + 1), S.mem);
    S.tileFirst = (u32 *)take(4 * maxTiles, S.mem);
    std::vector<std::pair<u64, u64>> tmp;
    u64 *bsum = (u64 *)take(8 * (nb + 1), tmp);
    if (!S.pscan || !S.tileFirst || !bsum) {
        give_back(tmp);
        return PERFT_ERR_OUT_OF_MEMORY;
    }
    k_scan_reduce<<<(unsigned)nb, SCAN_NT, 0, st>>>(S.L.cnt, n, bsum);
    k_scan_top<<<1, SCAN_TOP_NT, 0, st>>>(bsum, nb, S.pscan + n);
    k_scan_apply<<<(unsigned)nb, SCAN_NT, 0, st>>>(S.L.cnt, n, bsum, S.pscan, S.tileFirst, TILE_CAP_LOG2);
    launches += 3;
    // a table level's nodes leave the pending count in its finish pass
    if (!S.tt) {
        k_serve_zero_parents<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(S.L.cnt, S.L.root, n, pending);
        launches++;
    }
    give_back(tmp);
    if (cudaMemcpyAsync(hostTotal, S.pscan + n, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PERFT_ERR_CUDA;
    S.total = hostTotal[0];
    S.scanned = true;
    return PERFT_OK;
}

int Server::launch(int mode, ServeLevel &S, u64 lo, u64 hi, DeviceLevel *child)
{
    TileParams P;
    memset(&P, 0, sizeof P);
    P.ppl = S.L.planes;
    P.pstride = S.L.stride;
    P.pscan = S.pscan;
    P.proot = S.L.root;
    P.nParents = S.L.n;
    P.tileFirst = S.tileFirst;
    P.itemBase = lo;
    P.itemEnd = hi;
    P.capLog2 = TILE_CAP_LOG2;
    P.tileCounter = dCounter;
    if (child) {
        P.cpl = child->planes;
        P.cstride = child->stride;
        P.ccnt = child->cnt;
        P.croot = child->root;
    }
    P.rootCounts = counts;
    P.pending = pending;
    P.err = dErr;
    const u64 nTiles = (hi - lo + TILE_CAP - 1) / TILE_CAP;
    if (cudaMemsetAsync(dCounter, 0, 4, st) != cudaSuccess) return PERFT_ERR_CUDA;
    if (mode == MODE_LEAF && S.tt) {
        // sums per node (the parent's own slot of acc), as the engine's table levels do
        P.proot = nullptr;
        P.rootCounts = S.L.acc;
        P.pending = nullptr;
        launch_tile_variant<MODE_LEAF>(leafSplit ? SV_KOGGE_SPLIT : SV_KOGGE,
                                       (int)std::min<u64>(gridLeafAcc, nTiles), st, P);
    } else if (mode == MODE_EXPAND && S.tt) {
        // a table level expands without pending tracking; the children's
        // root entries are parent indices (their counts flow into its sums)
        P.proot = nullptr;
        P.pending = nullptr;
        launch_tile_variant<MODE_EXPAND>(SV_KOGGE, (int)std::min<u64>(gridExpandTT, nTiles), st, P);
    } else if (mode == MODE_LEAF && leafSplit)
        k_tile<MODE_LEAF, SV_KOGGE_SPLIT, true>
            <<<(int)std::min<u64>(gridLeaf, nTiles), TILE_NT, TILE_DYN_SMEM, st>>>(P);
    else if (mode == MODE_LEAF)
        k_tile<MODE_LEAF, SV_KOGGE, true><<<(int)std::min<u64>(gridLeaf, nTiles), TILE_NT, TILE_DYN_SMEM, st>>>(P);
    else
        k_tile<MODE_EXPAND, SV_KOGGE, true><<<(int)std::min<u64>(gridExpand, nTiles), TILE_NT, TILE_DYN_SMEM, st>>>(P);
    launches++;
    return cudaGetLastError() == cudaSuccess ? PERFT_OK : PERFT_ERR_CUDA;
}

int Server::advance()
{
    const u64 launchesBefore = launches;
    for (int r = 2; r <= SERVE_MAX_R; r++) {
        std::vector<ServeLevel *> keep;
        std::vector<ServeLevel *> work;
        work.swap(pools[r]);
        for (size_t li = 0; li < work.size(); li++) {
            ServeLevel *S = work[li];
            if (!S->scanned) {
                int rc = scan_level(*S);
                if (rc == PERFT_ERR_OUT_OF_MEMORY) {  // retry next iteration
                    keep.push_back(S);
                    continue;
                }
                if (rc != PERFT_OK) return rc;
            }
            u64 lo = S->next, hi = std::min(S->total, lo + stepItems);
            if (lo < hi) {
                if (r == 2) {
                    int rc = launch(MODE_LEAF, *S, lo, hi, nullptr);
                    if (rc != PERFT_OK) return rc;
                } else {
                    ServeLevel *C = nullptr;
                    for (;;) {  // shrink the step until the children fit
                        C = new ServeLevel();
                        C->r = r - 1;
                        const u64 m = hi - lo;
                        C->L.n = m;
                        C->L.stride = (m + 31) & ~31ULL;
                        C->L.planes = (u64 *)take(48 * C->L.stride, C->mem);
                        C->L.cnt = (u32 *)take(4 * C->L.stride, C->mem);
                        C->L.root = (u32 *)take(4 * C->L.stride, C->mem);
                        if (C->L.planes && C->L.cnt && C->L.root) break;
                        give_back(C->mem);
                        delete C;
                        C = nullptr;
                        if (hi - lo <= (u64)TILE_CAP) break;
                        hi = lo + (((hi - lo) / 2 + TILE_CAP - 1) & ~(u64)(TILE_CAP - 1));
                    }
                    if (!C) {  // no memory this iteration
                        keep.push_back(S);
                        continue;
                    }
                    int rc = launch(MODE_EXPAND, *S, lo, hi, &C->L);
                    if (rc != PERFT_OK) return rc;
                    if (S->tt) {
                        C->parent = S;
                        S->outstanding++;
                    }
                    pools[r - 1].push_back(C);
                }
                S->next = hi;
            }
            if (S->next >= S->total) {
                const int rc = retire(S);
                if (rc != PERFT_OK) return rc;
            } else {
                keep.push_back(S);
            }
        }
        for (ServeLevel *S : keep) pools[r].push_back(S);
    }
    // Levels that cannot get memory wait for others to finish; if nothing at
    // all could run for many iterations the budget is too small for the
    // admitted work: fail loudly instead of spinning.
    bool pendingWork = !waiting.empty();
    for (int r = 2; r <= SERVE_MAX_R; r++) pendingWork |= !pools[r].empty();
    idleIterations = (launches == launchesBefore && pendingWork) ? idleIterations + 1 : 0;
    return idleIterations > 200 ? PERFT_ERR_OUT_OF_MEMORY : PERFT_OK;
}

int Server::complete()
{
    if (!maxSlotUsed) return PERFT_OK;
    if (cudaMemcpyAsync(hostPending, pending, 8ull * maxSlotUsed, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(hostCounts, counts, 8ull * maxSlotUsed, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        (tt && cudaMemcpyAsync(hostTTStats, dTTStats, sizeof(TTStats), cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PERFT_ERR_CUDA;
    const double t = now_s();
    bool any = false;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (u32 s = 0; s < maxSlotUsed; s++) {
            ServeQuery *q = bySlot[s];
            if (!q || hostPending[s] != 0) continue;
            q->result = hostCounts[s];
            q->state = 2;
            q->tDone = t;
            bySlot[s] = nullptr;
            freeSlots.push_back(s);
            reserved -= q->predicted;
            inFlight--;
            completed++;
            any = true;
        }
        while (maxSlotUsed && !bySlot[maxSlotUsed - 1]) maxSlotUsed--;
    }
    if (any) cvDone.notify_all();
    return PERFT_OK;
}

void Server::loop()
{
    cudaSetDevice(dev);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cvWork.wait_for(lk, std::chrono::milliseconds(50),
                            [&] { return stopping || !queue.empty() || inFlight > 0; });
            if (stopping) break;
            if (queue.empty() && inFlight == 0) continue;
        }
        int rc = admit();
        if (rc == PERFT_OK) rc = advance();
        if (rc == PERFT_OK) rc = complete();
        iterations++;
        if (rc != PERFT_OK) {
            std::lock_guard<std::mutex> lk(mu);
            lastError = rc;
            break;
        }
    }
}

Server g_server;

}  // namespace
