// Host-side utilities of the C ABI: FEN parsing and printing, UCI move
// strings, divided perft, seeded playout positions.  They use the host build
// of the move generator for move lists only; every leaf count is computed by
// the GPU engine (engine.cu).
#include <algorithm>
#include <atomic>
#include <thread>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/file.h>
#include <unistd.h>

#include "../../include/perft_b200.h"
#include "movegen.cuh"

namespace pg {
void build_tables();
int engine_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out);
}  // namespace pg

using namespace pg;

namespace {

struct VecSink {
    std::vector<u32> *v;
    void operator()(u32 m) { v->push_back(m); }
};

std::vector<u32> legal_moves(const Board &b)
{
    std::vector<u32> v;
    v.reserve(64);
    VecSink s{&v};
    gen_moves<SV_KOGGE>(b, s);
    return v;
}

// Relative move -> UCI string (absolute squares).
void move_to_uci(const Board &b, u32 mv, char out[6])
{
    const bool black = (b.pawns >> 63) & 1;
    int from = mv & 63, to = (mv >> 6) & 63;
    const u32 fl = mv >> 12;
    if (black) {
        from ^= 56;
        to ^= 56;
    }
    out[0] = (char)('a' + (from & 7));
    out[1] = (char)('1' + (from >> 3));
    out[2] = (char)('a' + (to & 7));
    out[3] = (char)('1' + (to >> 3));
    if (fl & MF_PROMO) {
        out[4] = "nbrq"[fl & 3];
        out[5] = 0;
    } else {
        out[4] = 0;
    }
}

bool board_ok(const perft_pos48 *p) { return validate_pos48(p->bb) == 0; }

// Frontier of a deep search: the distinct side-relative boards a fixed number
// of plies below the root moves, each searched once however many move paths
// (from however many root moves) reach it.  This host-side transposition merge
// plays the role of the reference's complete hash tables for perft 11+
// (launcher.h:585-697); the side bit is dropped from the key because counts of
// a side-relative board do not depend on the real colour.
struct BoardKey {
    u64 w[6];
    bool operator==(const BoardKey &o) const { return memcmp(w, o.w, sizeof w) == 0; }
};
struct BoardKeyHash {
    size_t operator()(const BoardKey &k) const
    {
        u64 h = 0x9E3779B97F4A7C15ULL;
        for (u64 x : k.w) h = (h ^ x) * 0xBF58476D1CE4E5B9ULL;
        return (size_t)(h ^ (h >> 31));
    }
};

constexpr int MAX_MOVES_BUF = 256;  // more than the 218 legal moves any position has

struct ArraySink {
    u32 *m;
    u32 n;
    void operator()(u32 x) { m[n++] = x; }
};

using BoardCounts = std::unordered_map<BoardKey, u64, BoardKeyHash>;

BoardKey key_of(const Board &b) { return BoardKey{{b.mine, b.pawns & ~SIDE_BIT, b.knights, b.bq, b.rq, b.kings}}; }

// Distinct boards `plies` below b with the number of paths reaching each.
void enumerate_counts(const Board &b, u32 plies, BoardCounts &out)
{
    if (plies == 0) {
        out[key_of(b)] += 1;
        return;
    }
    u32 mv[MAX_MOVES_BUF];
    ArraySink sink{mv, 0};
    gen_moves<SV_KOGGE>(b, sink);
    for (u32 i = 0; i < sink.n; i++) enumerate_counts(make_child(b, mv[i]), plies - 1, out);
}

struct Frontier {
    std::unordered_map<BoardKey, u32, BoardKeyHash> index;
    std::vector<BoardKey> boards;
    // (distinct board, path count) per root move
    std::vector<std::vector<std::pair<u32, u64>>> paths;

    // Root moves are enumerated on all host cores, each into its own map;
    // the maps are then merged in root-move order, so the board order (which
    // the shards of a multi-process run rely on) does not depend on timing.
    void build(const Board &root, const std::vector<u32> &mv, u32 plies)
    {
        const size_t R = mv.size();
        std::vector<BoardCounts> local(R);
        std::atomic<size_t> next{0};
        std::atomic<bool> failed{false};
        // an exception must not leave a worker thread (that would terminate
        // the process): workers record it and the caller rethrows
        auto work = [&]() {
            try {
                for (size_t i; !failed && (i = next.fetch_add(1)) < R;)
                    enumerate_counts(make_child(root, mv[i]), plies, local[i]);
            } catch (...) {
                failed = true;
            }
        };
        unsigned T = std::max(1u, std::thread::hardware_concurrency());
        if (T > R) T = (unsigned)std::max<size_t>(R, 1);
        std::vector<std::thread> pool;
        try {
            for (unsigned t = 1; t < T; t++) pool.emplace_back(work);
        } catch (...) {
            // fewer threads than asked for: the started ones and this one finish the work
        }
        work();
        for (auto &t : pool) t.join();
        if (failed) throw std::bad_alloc();
        paths.assign(R, {});
        for (size_t i = 0; i < R; i++) {
            paths[i].reserve(local[i].size());
            for (const auto &kv : local[i]) {
                auto it = index.find(kv.first);
                u32 id;
                if (it == index.end()) {
                    id = (u32)boards.size();
                    index.emplace(kv.first, id);
                    boards.push_back(kv.first);
                } else {
                    id = it->second;
                }
                paths[i].emplace_back(id, kv.second);
            }
            BoardCounts().swap(local[i]);
        }
    }
};

// Counts of completed subtrees by (board, remaining depth), optionally backed
// by an append-only file.  Record: six board words (side bit cleared), the
// count, the depth and a check word over all of them; 64 bytes.
struct StoreRecord {
    u64 w[6];
    u64 count;
    u32 depth;
    u32 check;
};
static_assert(sizeof(StoreRecord) == 64, "store record is 64 bytes");
const char STORE_MAGIC[16] = "PERFTB200STORE1";

u32 record_check(const StoreRecord &r)
{
    u64 h = 0x243F6A8885A308D3ULL ^ r.depth;
    for (u64 x : r.w) h = (h ^ x) * 0x9E3779B97F4A7C15ULL;
    h = (h ^ r.count) * 0xD6E8FEB86659FD93ULL;
    h ^= h >> 32;
    return (u32)h ^ 0xA5A5A5A5u;
}

struct StoreKey {
    BoardKey b;
    u32 depth;
    bool operator==(const StoreKey &o) const { return depth == o.depth && b == o.b; }
};
struct StoreKeyHash {
    size_t operator()(const StoreKey &k) const { return BoardKeyHash()(k.b) ^ (k.depth * 0x9E3779B97F4A7C15ULL); }
};

struct ResultStore {
    std::mutex mu;
    bool open = false;
    int fd = -1;  // append-only descriptor of the backing file, or -1
    std::unordered_map<StoreKey, u64, StoreKeyHash> map;
    u64 hits = 0, appended = 0;
};
ResultStore g_store;

// Exclusive advisory lock on a store file for one scope.  Processes sharing
// a store (the shard processes of a multi-GPU run) take it around every
// append and around the open-time header write and tail repair, so no
// process sees another's half-written batch.  On a file system without
// lock support the scope runs unlocked: one process per store stays safe.
struct FileLock {
    int fd;
    bool locked = false, ok = false;
    explicit FileLock(int f) : fd(f)
    {
        int r;
        do {
            r = flock(fd, LOCK_EX);
        } while (r != 0 && errno == EINTR);
        locked = r == 0;
        ok = locked || errno == ENOLCK || errno == EOPNOTSUPP || errno == ENOSYS;
    }
    ~FileLock()
    {
        if (locked) flock(fd, LOCK_UN);
    }
};

bool write_all(int fd, const void *buf, size_t len)
{
    const char *p = (const char *)buf;
    while (len) {
        const ssize_t w = write(fd, p, len);
        if (w < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        p += w;
        len -= (size_t)w;
    }
    return true;
}

// Reads up to len bytes at off; returns the bytes read (short only at end
// of file) or -1.
ssize_t read_at(int fd, void *buf, size_t len, off_t off)
{
    char *p = (char *)buf;
    size_t got = 0;
    while (got < len) {
        const ssize_t r = pread(fd, p + got, len - got, off + (off_t)got);
        if (r < 0) {
            if (errno == EINTR) continue;
            return -1;
        }
        if (r == 0) break;
        got += (size_t)r;
    }
    return (ssize_t)got;
}

// Looks up every board of `ids` at `depth`; found ones go to counts and are
// removed from ids.
void store_lookup(const Frontier &f, u32 depth, std::vector<u32> &ids, std::vector<u64> &counts)
{
    std::lock_guard<std::mutex> lk(g_store.mu);
    if (!g_store.open) return;
    size_t k = 0;
    for (u32 id : ids) {
        auto it = g_store.map.find(StoreKey{f.boards[id], depth});
        if (it != g_store.map.end()) {
            counts[id] = it->second;
            g_store.hits++;
        } else {
            ids[k++] = id;
        }
    }
    ids.resize(k);
}

int store_add(const Frontier &f, u32 depth, const u32 *ids, const u64 *vals, u32 n)
{
    std::lock_guard<std::mutex> lk(g_store.mu);
    if (!g_store.open) return PERFT_OK;
    std::vector<StoreRecord> recs;
    recs.reserve(n);
    for (u32 i = 0; i < n; i++) {
        const BoardKey &b = f.boards[ids[i]];
        if (!g_store.map.emplace(StoreKey{b, depth}, vals[i]).second) continue;
        StoreRecord r;
        memcpy(r.w, b.w, sizeof r.w);
        r.count = vals[i];
        r.depth = depth;
        r.check = record_check(r);
        recs.push_back(r);
    }
    if (g_store.fd >= 0 && !recs.empty()) {
        // one write of whole records at the end of the file (O_APPEND) under
        // the file lock; a failed write is cut back so that later appends,
        // from this or another process, stay on record boundaries
        FileLock lock(g_store.fd);
        if (!lock.ok) return PERFT_ERR_IO;
        const off_t end = lseek(g_store.fd, 0, SEEK_END);
        if (end < 0) return PERFT_ERR_IO;
        if (!write_all(g_store.fd, recs.data(), recs.size() * sizeof(StoreRecord))) {
            if (ftruncate(g_store.fd, end) != 0) { /* the next open drops the torn tail */ }
            return PERFT_ERR_IO;
        }
        g_store.appended += recs.size();
    }
    return PERFT_OK;
}

// perft(depth) of the distinct frontier boards whose index is congruent to
// `shard` modulo `n_shards`, in GPU batches; the others are left at 0.
int frontier_counts(const Frontier &f, u32 depth, u32 shard, u32 n_shards, std::vector<u64> &counts)
{
    constexpr u32 CHUNK = 1u << 18;
    const u32 total = (u32)f.boards.size();
    counts.assign(total, 0);
    std::vector<u32> ids;
    for (u32 i = shard; i < total; i += n_shards) ids.push_back(i);
    store_lookup(f, depth, ids, counts);
    std::vector<u64> pos, out;
    std::vector<uint8_t> depths;
    for (size_t lo = 0; lo < ids.size(); lo += CHUNK) {
        const u32 n = (u32)std::min<size_t>(CHUNK, ids.size() - lo);
        pos.resize(6ull * n);
        for (u32 i = 0; i < n; i++) {
            Board b;
            memcpy(&b, f.boards[ids[lo + i]].w, sizeof b);
            to_pos48(b, &pos[6ull * i]);
        }
        depths.assign(n, (uint8_t)depth);
        out.assign(n, 0);
        const int rc = engine_batch_host(pos.data(), depths.data(), n, out.data());
        if (rc != PERFT_OK) return rc;
        for (u32 i = 0; i < n; i++) counts[ids[lo + i]] = out[i];
        const int src = store_add(f, depth, ids.data() + lo, out.data(), n);
        if (src != PERFT_OK) return src;
    }
    return PERFT_OK;
}

// The frontier of the last sharded deep call.  A rank that takes several
// shards of one deep search in turn (dynamic dealing: shard j of n as the
// shared cursor hands them out) builds the frontier once; the enumeration is
// deterministic, so the cached frontier is the one a rebuild would give.
// Unsharded calls neither use nor keep it (a frontier can hold gigabytes).
struct FrontierCache {
    std::mutex mu;
    u64 root[6] = {};
    u32 plies = 0;
    std::shared_ptr<const Frontier> f;
} g_frontierCache;

std::shared_ptr<const Frontier> frontier_for(const perft_pos48 *pos, const Board &b, const std::vector<u32> &mv,
                                             u32 plies, bool sharded)
{
    if (!sharded) {
        std::lock_guard<std::mutex> lk(g_frontierCache.mu);
        g_frontierCache.f.reset();
    } else {
        std::lock_guard<std::mutex> lk(g_frontierCache.mu);
        if (g_frontierCache.f && g_frontierCache.plies == plies &&
            memcmp(g_frontierCache.root, pos->bb, sizeof g_frontierCache.root) == 0)
            return g_frontierCache.f;
    }
    auto f = std::make_shared<Frontier>();
    f->build(b, mv, plies);
    if (sharded) {
        std::lock_guard<std::mutex> lk(g_frontierCache.mu);
        memcpy(g_frontierCache.root, pos->bb, sizeof g_frontierCache.root);
        g_frontierCache.plies = plies;
        g_frontierCache.f = f;
    }
    return f;
}

// C-ABI functions return status codes: an exception (host memory
// exhausted) must not cross the boundary.
template <class F>
int guarded(F f)
{
    try {
        return f();
    } catch (const std::bad_alloc &) {
        return PERFT_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return PERFT_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

// Utils::readFENString (util.cpp:189-281) then board088ToHexBB
// (util.cpp:92-140): placement, side, castling letters, en-passant file;
// clocks are not read.
int perft_fen_to_pos(const char *fen, perft_pos48 *out)
{
    if (!fen || !out) return PERFT_ERR_INVALID_ARG;
    build_tables();
    u64 bb[6] = {0, 0, 0, 0, 0, 0};
    int i = 0, row = 0, col = 0;
    for (; fen[i]; i++) {
        const char ch = fen[i];
        if (ch == '/' || ch == '\\') {
            row++;
            col = 0;
        } else if (ch >= '1' && ch <= '8') {
            col += ch - '0';
        } else if (strchr("kqrbnpKQRBNP", ch)) {
            if (row > 7 || col > 7) return PERFT_ERR_BAD_FEN;
            const u64 bit = 1ULL << ((7 - row) * 8 + col);
            if (ch >= 'A' && ch <= 'Z') bb[0] |= bit;
            switch (ch | 0x20) {
            case 'p': bb[1] |= bit; break;
            case 'n': bb[2] |= bit; break;
            case 'b': bb[3] |= bit; break;
            case 'r': bb[4] |= bit; break;
            case 'q': bb[3] |= bit; bb[4] |= bit; break;
            case 'k': bb[5] |= bit; break;
            }
            col++;
        } else if (ch == ' ') {
            break;
        } else {
            return PERFT_ERR_BAD_FEN;
        }
        if (row >= 7 && col == 8) break;
    }
    if (!fen[i]) return PERFT_ERR_BAD_FEN;
    if (bb[1] & ~RANKS2TO7) return PERFT_ERR_BAD_FEN;
    i++;
    while (fen[i] == ' ') i++;
    const int black = (fen[i] == 'b' || fen[i] == 'B') ? 1 : 0;
    if (fen[i]) i++;
    while (fen[i] == ' ') i++;
    u64 wc = 0, bc = 0;
    while (fen[i] && fen[i] != ' ') {
        switch (fen[i]) {
        case 'k': bc |= 1; break;
        case 'q': bc |= 2; break;
        case 'K': wc |= 1; break;
        case 'Q': wc |= 2; break;
        }
        i++;
    }
    while (fen[i] == ' ') i++;
    u64 ep = 0;
    if (fen[i] >= 'a' && fen[i] <= 'h') ep = (u64)(fen[i] - 'a' + 1);
    bb[1] |= wc | (bc << 2) | (ep << 4) | ((u64)black << 63);
    memcpy(out->bb, bb, sizeof bb);
    return validate_pos48(bb) == 0 ? PERFT_OK : PERFT_ERR_BAD_FEN;
}

int perft_pos_to_fen(const perft_pos48 *pos, char *buf, size_t len)
{
    if (!pos || !buf || len < 2) return PERFT_ERR_INVALID_ARG;
    const u64 *p = pos->bb;
    const u64 pawns = p[1] & RANKS2TO7;
    std::string s;
    for (int r = 7; r >= 0; r--) {
        int empty = 0;
        for (int f = 0; f < 8; f++) {
            const u64 bit = 1ULL << (r * 8 + f);
            char c = 0;
            if (pawns & bit) c = 'p';
            else if (p[2] & bit) c = 'n';
            else if ((p[3] & p[4]) & bit) c = 'q';
            else if (p[3] & bit) c = 'b';
            else if (p[4] & bit) c = 'r';
            else if (p[5] & bit) c = 'k';
            if (!c) {
                empty++;
                continue;
            }
            if (empty) s += (char)('0' + empty);
            empty = 0;
            if (p[0] & bit) c = (char)(c - 32);
            s += c;
        }
        if (empty) s += (char)('0' + empty);
        if (r) s += '/';
    }
    const bool black = (p[1] >> 63) & 1;
    s += black ? " b " : " w ";
    std::string cs;
    if (p[1] & 1) cs += 'K';
    if (p[1] & 2) cs += 'Q';
    if (p[1] & 4) cs += 'k';
    if (p[1] & 8) cs += 'q';
    s += cs.empty() ? "-" : cs;
    const int ep = (int)((p[1] >> 4) & 15);
    if (ep) {
        s += ' ';
        s += (char)('a' + ep - 1);
        s += black ? '3' : '6';
    } else {
        s += " -";
    }
    s += " 0 1";
    if (s.size() + 1 > len) return PERFT_ERR_INVALID_ARG;
    memcpy(buf, s.c_str(), s.size() + 1);
    return PERFT_OK;
}

int perft_legal_moves_uci(const perft_pos48 *pos, char *buf, size_t len, uint32_t *n_moves)
{
    if (!pos || !buf || !len) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    build_tables();
    const Board b = from_pos48(pos->bb);
    const std::vector<u32> mv = legal_moves(b);
    std::string s;
    for (size_t i = 0; i < mv.size(); i++) {
        char u[6];
        move_to_uci(b, mv[i], u);
        if (i) s += ' ';
        s += u;
    }
    if (s.size() + 1 > len) return PERFT_ERR_INVALID_ARG;
    memcpy(buf, s.c_str(), s.size() + 1);
    if (n_moves) *n_moves = (uint32_t)mv.size();
    return PERFT_OK;
}

int perft_apply_uci_move(perft_pos48 *pos, const char *uci)
{
    if (!pos || !uci) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    build_tables();
    const Board b = from_pos48(pos->bb);
    for (u32 m : legal_moves(b)) {
        char u[6];
        move_to_uci(b, m, u);
        if (strcmp(u, uci) == 0) {
            to_pos48(make_child(b, m), pos->bb);
            return PERFT_OK;
        }
    }
    return PERFT_ERR_ILLEGAL_MOVE;
}

static int divide_impl(const perft_pos48 *pos, uint32_t depth, char (*moves)[6], uint64_t *counts,
                 uint32_t *n_moves)
{
    if (!pos || !moves || !counts || !n_moves || depth < 1 || depth > 21) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    build_tables();
    const Board b = from_pos48(pos->bb);
    const std::vector<u32> mv = legal_moves(b);
    std::vector<u64> children(6 * mv.size());
    std::vector<uint8_t> depths(mv.size(), (uint8_t)(depth - 1));
    for (size_t i = 0; i < mv.size(); i++) {
        to_pos48(make_child(b, mv[i]), &children[6 * i]);
        move_to_uci(b, mv[i], moves[i]);
    }
    *n_moves = (uint32_t)mv.size();
    if (mv.empty()) return PERFT_OK;
    return engine_batch_host(children.data(), depths.data(), (u32)mv.size(), counts);
}

int perft_random_playouts(uint64_t seed, uint32_t n, uint32_t min_plies, uint32_t max_plies,
                          perft_pos48 *out)
{
    if ((!out && n) || min_plies > max_plies || max_plies > 1000) return PERFT_ERR_INVALID_ARG;
    build_tables();
    std::mt19937_64 rng(seed);
    perft_pos48 start;
    perft_fen_to_pos("rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", &start);
    uint32_t made = 0;
    while (made < n) {
        const uint32_t plies =
            min_plies + (uint32_t)(rng() % (uint64_t)(max_plies - min_plies + 1));
        Board b = from_pos48(start.bb);
        bool ok = true;
        for (uint32_t k = 0; k < plies; k++) {
            const std::vector<u32> mv = legal_moves(b);
            if (mv.empty()) {
                ok = false;
                break;
            }
            b = make_child(b, mv[rng() % mv.size()]);
        }
        if (!ok || count_moves<SV_KOGGE>(b) == 0) continue;
        to_pos48(b, out[made].bb);
        made++;
    }
    return PERFT_OK;
}

// Deep perft by host root split: the distinct positions `split_plies` below
// the root moves are merged across all root moves and searched once each on
// the GPU at the remaining depth; per-move subtotals weight each board's count
// by its path count.  They are the divided perft the reference prints for deep
// runs (launcher.h:1181-1450).  split_plies is clamped to depth - 1.  With
// n_shards > 1 only every n_shards-th frontier board (from `shard`) is
// searched, so the per-move subtotals of shards 0..n_shards-1 sum to the full
// result: the multi-GPU root split, one process per GPU (launcher.h:476-583).
static int deep_shard_impl(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint32_t shard,
                     uint32_t n_shards, char (*moves)[6], uint64_t *counts, uint32_t *n_moves, uint64_t *total)
{
    if (!pos || !total || depth < 1 || depth > 30) return PERFT_ERR_INVALID_ARG;
    if (n_shards == 0 || shard >= n_shards) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    if (split_plies + 1 > depth) split_plies = depth - 1;
    if (depth - 1 - split_plies > 20) return PERFT_ERR_INVALID_ARG;
    build_tables();
    const Board b = from_pos48(pos->bb);
    const std::vector<u32> mv = legal_moves(b);
    std::shared_ptr<const Frontier> fp;
    try {
        fp = frontier_for(pos, b, mv, split_plies, n_shards > 1);
    } catch (const std::exception &) {
        return PERFT_ERR_OUT_OF_MEMORY;  // host memory or threads exhausted
    }
    const Frontier &f = *fp;
    std::vector<u64> sub;
    const int rc = frontier_counts(f, depth - 1 - split_plies, shard, n_shards, sub);
    if (rc != PERFT_OK) return rc;
    // 128-bit sums: a per-move subtotal must fit 64 bits; a total that does
    // not (perft 14 of the initial position and beyond) is reported as
    // PERFT_ERR_OVERFLOW with the subtotals filled in
    unsigned __int128 sum = 0;
    for (size_t i = 0; i < mv.size(); i++) {
        unsigned __int128 s = 0;
        for (const auto &kv : f.paths[i]) s += (unsigned __int128)sub[kv.first] * kv.second;
        if (s >> 64) {
            if (n_moves) *n_moves = 0;  // no usable subtotals
            return PERFT_ERR_OVERFLOW;
        }
        if (moves) move_to_uci(b, mv[i], moves[i]);
        if (counts) counts[i] = (u64)s;
        sum += s;
    }
    if (n_moves) *n_moves = (uint32_t)mv.size();
    *total = (u64)sum;
    return (sum >> 64) ? PERFT_ERR_OVERFLOW : PERFT_OK;
}

int perft_deep(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, char (*moves)[6],
               uint64_t *counts, uint32_t *n_moves, uint64_t *total)
{
    return perft_deep_shard(pos, depth, split_plies, 0, 1, moves, counts, n_moves, total);
}

// Size of the frontier perft_deep(pos, depth, split_plies) would search: the
// distinct boards 1 + split_plies plies below pos and the move paths that
// reach them.  Host only: for planning a deep run's memory and time.
static int deep_frontier_impl(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint64_t *n_boards,
                        uint64_t *n_paths)
{
    if (!pos || depth < 1 || depth > 30) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    if (split_plies + 1 > depth) split_plies = depth - 1;
    build_tables();
    const Board b = from_pos48(pos->bb);
    const std::vector<u32> mv = legal_moves(b);
    Frontier f;
    try {
        f.build(b, mv, split_plies);
    } catch (const std::exception &) {
        return PERFT_ERR_OUT_OF_MEMORY;
    }
    u64 paths = 0;
    for (const auto &root : f.paths)
        for (const auto &kv : root) paths += kv.second;
    if (n_boards) *n_boards = f.boards.size();
    if (n_paths) *n_paths = paths;
    return PERFT_OK;
}

static int store_open_impl(const char *path)
{
    std::lock_guard<std::mutex> lk(g_store.mu);
    if (g_store.fd >= 0) close(g_store.fd);
    g_store.fd = -1;
    g_store.map.clear();
    g_store.hits = g_store.appended = 0;
    g_store.open = false;
    if (!path) {
        g_store.open = true;
        return PERFT_OK;
    }
    const int fd = open(path, O_RDWR | O_CREAT | O_APPEND | O_CLOEXEC, 0644);
    if (fd < 0) return PERFT_ERR_IO;
    auto fail = [&]() {
        close(fd);
        g_store.map.clear();
        return PERFT_ERR_IO;
    };
    {
        FileLock lock(fd);
        if (!lock.ok) return fail();
        char head[64];
        const ssize_t got = read_at(fd, head, sizeof head, 0);
        if (got == 0) {
            memset(head, 0, sizeof head);
            memcpy(head, STORE_MAGIC, sizeof STORE_MAGIC);
            if (!write_all(fd, head, sizeof head)) return fail();
        } else if (got != (ssize_t)sizeof head || memcmp(head, STORE_MAGIC, sizeof STORE_MAGIC) != 0) {
            return fail();
        }
        off_t good = (off_t)sizeof head;
        std::vector<StoreRecord> buf(4096);
        for (bool more = true; more;) {
            const ssize_t r = read_at(fd, buf.data(), buf.size() * sizeof(StoreRecord), good);
            if (r < 0) return fail();
            const size_t k = (size_t)r / sizeof(StoreRecord);
            more = k == buf.size();
            for (size_t i = 0; i < k; i++) {
                const StoreRecord &rec = buf[i];
                if (record_check(rec) != rec.check) {
                    more = false;
                    break;
                }
                BoardKey b;
                memcpy(b.w, rec.w, sizeof b.w);
                g_store.map[StoreKey{b, rec.depth}] = rec.count;
                good += (off_t)sizeof rec;
            }
        }
        // drop a torn or corrupt tail so that appends continue after the last good record
        const off_t size = lseek(fd, 0, SEEK_END);
        if (size < 0 || (size > good && ftruncate(fd, good) != 0)) return fail();
    }
    g_store.fd = fd;
    g_store.open = true;
    return PERFT_OK;
}

int perft_result_store_close(void)
{
    std::lock_guard<std::mutex> lk(g_store.mu);
    int rc = PERFT_OK;
    if (g_store.fd >= 0 && close(g_store.fd) != 0) rc = PERFT_ERR_IO;
    g_store.fd = -1;
    g_store.map.clear();
    g_store.open = false;
    return rc;
}

int perft_result_store_stats(uint64_t *entries, uint64_t *hits, uint64_t *appended)
{
    std::lock_guard<std::mutex> lk(g_store.mu);
    if (!g_store.open) return PERFT_ERR_NOT_INITIALIZED;
    if (entries) *entries = g_store.map.size();
    if (hits) *hits = g_store.hits;
    if (appended) *appended = g_store.appended;
    return PERFT_OK;
}

// Records mode (launcher.h:1579-1695): every line of `in_path` is a FEN
// followed by an occurrence count; "<line> <perft> <perft x count>" is
// appended to "<in_path>.op".  Lines already present in the output are
// skipped, so an interrupted run resumes where it stopped.  Lines are
// searched in GPU batches of `batch` records.
// Records finished by an earlier run: the complete ('\n'-terminated) lines
// of the output file, whatever their length.  A torn last line (a run
// stopped in the middle of a write) is cut off, so its record is searched
// again instead of being skipped.
static int finished_records(const std::string &opPath, size_t *done)
{
    *done = 0;
    FILE *fo = fopen(opPath.c_str(), "rb");
    if (!fo) return PERFT_OK;  // no output yet
    off_t size = 0, complete = 0;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, fo)) > 0) {
        for (size_t i = 0; i < got; i++) {
            if (buf[i] == '\n') {
                (*done)++;
                complete = size + (off_t)i + 1;
            }
        }
        size += (off_t)got;
    }
    const bool failed = ferror(fo) != 0;
    fclose(fo);
    if (failed) return PERFT_ERR_IO;
    if (complete != size && truncate(opPath.c_str(), complete) != 0) return PERFT_ERR_IO;
    return PERFT_OK;
}

static int records_impl(const char *in_path, uint32_t depth, uint32_t batch, uint64_t *records_done)
{
    if (!in_path || depth > 20) return PERFT_ERR_INVALID_ARG;
    if (!batch) batch = 4096;
    if (records_done) *records_done = 0;
    FILE *fin = fopen(in_path, "r");
    if (!fin) return PERFT_ERR_NOT_FOUND;
    const std::string opPath = std::string(in_path) + ".op";
    size_t already = 0;
    if (const int frc = finished_records(opPath, &already); frc != PERFT_OK) {
        fclose(fin);
        return frc;
    }
    FILE *fout = fopen(opPath.c_str(), "a");
    if (!fout) {
        fclose(fin);
        return PERFT_ERR_IO;
    }
    std::vector<std::string> lines;
    std::vector<u64> pos, occ;
    u64 done = 0;
    int rc = PERFT_OK;
    auto flush = [&]() -> int {
        const u32 n = (u32)lines.size();
        if (!n) return PERFT_OK;
        std::vector<uint8_t> depths(n, (uint8_t)depth);
        std::vector<u64> out(n);
        const int r = engine_batch_host(pos.data(), depths.data(), n, out.data());
        if (r != PERFT_OK) return r;
        for (u32 i = 0; i < n; i++)
            fprintf(fout, "%s %llu %llu\n", lines[i].c_str(), (unsigned long long)out[i],
                    (unsigned long long)(out[i] * occ[i]));
        if (fflush(fout) != 0 || ferror(fout)) return PERFT_ERR_IO;
        done += n;
        lines.clear();
        pos.clear();
        occ.clear();
        return PERFT_OK;
    };
    char line[2048];
    size_t idx = 0;
    while (fgets(line, sizeof line, fin)) {
        size_t len = strlen(line);
        while (len && (line[len - 1] == '\n' || line[len - 1] == '\r')) line[--len] = 0;
        if (!len) continue;
        if (idx++ < already) continue;
        const char *sp = strrchr(line, ' ');
        const u64 count = sp ? strtoull(sp + 1, nullptr, 10) : 1;
        perft_pos48 p;
        if (perft_fen_to_pos(line, &p) != PERFT_OK) {
            rc = PERFT_ERR_BAD_FEN;
            break;
        }
        lines.emplace_back(line);
        pos.insert(pos.end(), p.bb, p.bb + 6);
        occ.push_back(count);
        if (lines.size() == batch && (rc = flush()) != PERFT_OK) break;
    }
    if (rc == PERFT_OK) rc = flush();
    fclose(fin);
    fclose(fout);
    if (records_done) *records_done = done;
    return rc;
}

// Feature bits of a position used to stratify synthetic workloads:
//   1 a legal en-passant capture exists, 2 the side to move has a pawn on
//   its 7th rank, 4 some castling right remains, 8 the side to move is in
//   check, 16 a promotion move exists.
int perft_position_features(const perft_pos48 *pos, uint32_t *features)
{
    if (!pos || !features) return PERFT_ERR_INVALID_ARG;
    if (!board_ok(pos)) return PERFT_ERR_INVALID_ARG;
    build_tables();
    const Board b = from_pos48(pos->bb);
    uint32_t f = 0;
    for (u32 m : legal_moves(b)) {
        if ((m >> 12) == MF_EP) f |= 1;
        if ((m >> 12) & MF_PROMO) f |= 16;
    }
    if (b.pawns & b.mine & RANKS2TO7 & 0x00FF000000000000ULL) f |= 2;
    if (b.pawns & 0x0F) f |= 4;
    Ctx c;
    setup_ctx<SV_KOGGE>(b, c);
    if (c.attacked & c.myK) f |= 8;
    *features = f;
    return PERFT_OK;
}

int perft_divide(const perft_pos48 *pos, uint32_t depth, char (*moves)[6], uint64_t *counts, uint32_t *n_moves)
{
    return guarded([&] { return divide_impl(pos, depth, moves, counts, n_moves); });
}

int perft_deep_shard(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint32_t shard,
                     uint32_t n_shards, char (*moves)[6], uint64_t *counts, uint32_t *n_moves, uint64_t *total)
{
    return guarded(
        [&] { return deep_shard_impl(pos, depth, split_plies, shard, n_shards, moves, counts, n_moves, total); });
}

int perft_deep_frontier(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint64_t *n_boards,
                        uint64_t *n_paths)
{
    return guarded([&] { return deep_frontier_impl(pos, depth, split_plies, n_boards, n_paths); });
}

int perft_result_store_open(const char *path)
{
    return guarded([&] { return store_open_impl(path); });
}

int perft_records(const char *in_path, uint32_t depth, uint32_t batch, uint64_t *records_done)
{
    return guarded([&] { return records_impl(in_path, depth, batch, records_done); });
}

}  // extern "C"
