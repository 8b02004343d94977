// Test infrastructure: a thin C-ABI driver around the REFERENCE's own host perft.
//
// This file is compiled together with the reference's unmodified host sources
// (GlobalVars.cpp, Magics.cpp, randoms.cpp, util.cpp and the headers
// MoveGeneratorBitboard.h / chess.h / switches.h) by oracle/Makefile into
// oracle/_ref/libperft_ref.so.  Nothing from the reference is copied here: the
// reference headers are #included from the reference tree at build time.
//
// It is the parity anchor for the clean-room oracle (oracle/perft_oracle.c)
// and the "reference" CPU baseline of bench.py.  Only tests/, the smoke check
// and bench.py's CPU-baseline leg load it; the product never does.
//
// Entry points mirror the reference's host routines:
//   ref_perft        -> perft_bb()                 perft_bb.h:79-101
//                       (generateBoards recursion, countMoves at depth 1)
//   ref_perft_gm     -> the GPU path's shape: generateMoves + makeMove +
//                       countMoves (perft_bb.h:412-446 leaf pass,
//                       perft_bb.h:601-625 level expansion)
//   ref_fen_to_pos   -> Utils::readFENString + Utils::board088ToHexBB
//                       (util.cpp:189-281, util.cpp:92-140)
//   ref_perft_mt     -> perft_bb, root-split over a thread pool (the CPU
//                       baseline: all host cores, summed per thread)

#include <stdint.h>
#include <string.h>
#include <atomic>
#include <thread>
#include <vector>

#include "MoveGeneratorBitboard.h"

static_assert(sizeof(HexaBitBoardPosition) == 48, "pos48 layout");

namespace {

bool g_ready = false;

uint32 countMovesAny(HexaBitBoardPosition *pos)
{
    // perft_bb.h:35-54 (template dispatch on side to move)
    if (pos->chance == BLACK)
        return MoveGeneratorBitboard::countMoves<BLACK>(pos);
    return MoveGeneratorBitboard::countMoves<WHITE>(pos);
}

uint32 generateBoardsAny(HexaBitBoardPosition *pos, HexaBitBoardPosition *out)
{
    // perft_bb.h:56-74
    if (pos->chance == BLACK)
        return MoveGeneratorBitboard::generateBoards<BLACK>(pos, out);
    return MoveGeneratorBitboard::generateBoards<WHITE>(pos, out);
}

uint32 generateMovesAny(HexaBitBoardPosition *pos, CMove *out)
{
    if (pos->chance == BLACK)
        return MoveGeneratorBitboard::generateMoves<BLACK>(pos, out);
    return MoveGeneratorBitboard::generateMoves<WHITE>(pos, out);
}

void makeMoveAny(HexaBitBoardPosition *pos, CMove m)
{
    uint64 unusedHash = 0;
    if (pos->chance == BLACK)
        MoveGeneratorBitboard::makeMove<BLACK, false>(pos, unusedHash, m);
    else
        MoveGeneratorBitboard::makeMove<WHITE, false>(pos, unusedHash, m);
}

// perft_bb.h:79-101, called the same way (countMoves at depth 1).
uint64 perftBB(HexaBitBoardPosition *pos, uint32 depth)
{
    if (depth == 0)
        return 1;
    if (depth == 1)
        return countMovesAny(pos);
    HexaBitBoardPosition children[MAX_MOVES];
    uint32 n = generateBoardsAny(pos, children);
    uint64 total = 0;
    for (uint32 i = 0; i < n; i++)
        total += perftBB(&children[i], depth - 1);
    return total;
}

// generateMoves + makeMove + countMoves: the shape of the reference GPU BFS.
uint64 perftGM(HexaBitBoardPosition *pos, uint32 depth)
{
    if (depth == 0)
        return 1;
    if (depth == 1)
        return countMovesAny(pos);
    CMove moves[MAX_MOVES];
    uint32 n = generateMovesAny(pos, moves);
    uint64 total = 0;
    for (uint32 i = 0; i < n; i++) {
        HexaBitBoardPosition child = *pos;
        makeMoveAny(&child, moves[i]);
        total += perftGM(&child, depth - 1);
    }
    return total;
}

struct Task {
    HexaBitBoardPosition pos;
    uint32 depth;
    uint32 owner;   // index of the root position this subtree belongs to
};

// Root-split: expand each root two plies (or fewer for shallow depths) into
// independent subtree tasks, then let all threads pull tasks from a shared
// atomic cursor and sum into per-thread, per-root accumulators.
void splitRoots(const HexaBitBoardPosition *roots, const uint32_t *depths, uint32_t n,
                std::vector<Task> &tasks, std::vector<uint64> &direct)
{
    for (uint32_t r = 0; r < n; r++) {
        HexaBitBoardPosition root = roots[r];
        uint32 d = depths[r];
        if (d <= 3) {
            tasks.push_back({root, d, r});
            continue;
        }
        HexaBitBoardPosition c1[MAX_MOVES];
        uint32 n1 = generateBoardsAny(&root, c1);
        for (uint32 i = 0; i < n1; i++) {
            HexaBitBoardPosition c2[MAX_MOVES];
            uint32 n2 = generateBoardsAny(&c1[i], c2);
            for (uint32 j = 0; j < n2; j++)
                tasks.push_back({c2[j], d - 2, r});
        }
    }
    (void)direct;
}

}  // namespace

extern "C" {

int ref_init(void)
{
    if (!g_ready) {
        MoveGeneratorBitboard::init();
        g_ready = true;
    }
    return 0;
}

int ref_fen_to_pos(const char *fen, uint64_t out[6])
{
    ref_init();
    char buf[1024];
    size_t len = strlen(fen);
    if (len >= sizeof(buf) - 2)
        return -1;
    memcpy(buf, fen, len + 1);
    BoardPosition b88;
    Utils::readFENString(buf, &b88);
    HexaBitBoardPosition hb;
    Utils::board088ToHexBB(&hb, &b88);
    memcpy(out, &hb, sizeof(hb));
    return 0;
}

uint32_t ref_count_moves(const uint64_t pos[6])
{
    ref_init();
    HexaBitBoardPosition p;
    memcpy(&p, pos, sizeof(p));
    return countMovesAny(&p);
}

// Children as produced by the reference's generateBoards (full boards).
uint32_t ref_children(const uint64_t pos[6], uint64_t *out /* [MAX_MOVES][6] */)
{
    ref_init();
    HexaBitBoardPosition p;
    memcpy(&p, pos, sizeof(p));
    HexaBitBoardPosition children[MAX_MOVES];
    uint32 n = generateBoardsAny(&p, children);
    memcpy(out, children, sizeof(HexaBitBoardPosition) * n);
    return n;
}

uint64_t ref_perft(const uint64_t pos[6], uint32_t depth)
{
    ref_init();
    HexaBitBoardPosition p;
    memcpy(&p, pos, sizeof(p));
    return perftBB(&p, depth);
}

uint64_t ref_perft_gm(const uint64_t pos[6], uint32_t depth)
{
    ref_init();
    HexaBitBoardPosition p;
    memcpy(&p, pos, sizeof(p));
    return perftGM(&p, depth);
}

// Multi-threaded batch perft (root split).  out[i] = perft(pos[i], depths[i]).
int ref_perft_batch_mt(const uint64_t *pos, const uint32_t *depths, uint32_t n,
                       int threads, uint64_t *out)
{
    ref_init();
    if (threads < 1)
        threads = 1;
    std::vector<HexaBitBoardPosition> roots(n);
    memcpy(roots.data(), pos, sizeof(HexaBitBoardPosition) * n);
    std::vector<Task> tasks;
    std::vector<uint64> direct;
    splitRoots(roots.data(), depths, n, tasks, direct);

    std::atomic<size_t> cursor(0);
    std::vector<std::vector<uint64>> partial(threads, std::vector<uint64>(n, 0));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([&, t]() {
            for (;;) {
                size_t i = cursor.fetch_add(1);
                if (i >= tasks.size())
                    break;
                Task task = tasks[i];
                partial[t][task.owner] += perftBB(&task.pos, task.depth);
            }
        });
    }
    for (auto &th : pool)
        th.join();
    for (uint32_t r = 0; r < n; r++) {
        uint64 s = 0;
        for (int t = 0; t < threads; t++)
            s += partial[t][r];
        out[r] = s;
    }
    return 0;
}

uint64_t ref_perft_mt(const uint64_t pos[6], uint32_t depth, int threads)
{
    uint64_t out = 0;
    ref_perft_batch_mt(pos, &depth, 1, threads, &out);
    return out;
}

}  // extern "C"
