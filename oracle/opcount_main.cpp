// Test infrastructure: measures the average number of 64-bit integer
// operations the restated reference algorithm spends per countMoves,
// generateMoves and makeMove call, over the perft trees of the positions in
// a pos48 file.  Output: one JSON object on stdout.
//
//   opcount <positions.bin> <depth>
//
// The trees are walked exactly as the GPU path does (generate + make at
// interior plies, countMoves at the last ply).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "perft_oracle.c"

uint64_t g_ops = 0;

static uint64_t n_count = 0, ops_count = 0, n_gen = 0, ops_gen = 0, n_make = 0, ops_make = 0;
static uint64_t gen_moves_total = 0;

static uint64_t walk(const oracle_pos *pos, uint32_t depth)
{
    if (depth == 1) {
        uint64_t o = g_ops;
        uint32_t c = oracle_count_moves(pos);
        ops_count += g_ops - o;
        n_count++;
        return c;
    }
    uint16_t moves[256];
    uint64_t o = g_ops;
    uint32_t n = oracle_generate_moves(pos, moves);
    ops_gen += g_ops - o;
    n_gen++;
    gen_moves_total += n;
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) {
        oracle_pos child = *pos;
        o = g_ops;
        oracle_make_move(&child, moves[i]);
        ops_make += g_ops - o;
        n_make++;
        total += walk(&child, depth - 1);
    }
    return total;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: opcount <positions.bin> <depth>\n");
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<oracle_pos> pos;
    oracle_pos p;
    while (fread(&p, sizeof p, 1, f) == 1) pos.push_back(p);
    fclose(f);
    const uint32_t depth = (uint32_t)atoi(argv[2]);
    oracle_init();
    g_ops = 0;
    uint64_t leaves = 0;
    for (auto &q : pos) leaves += walk(&q, depth);
    printf("{\"positions\": %zu, \"depth\": %u, \"leaves\": %llu, "
           "\"count_calls\": %llu, \"c_count\": %.3f, "
           "\"gen_calls\": %llu, \"c_gen\": %.3f, \"moves_per_gen\": %.3f, "
           "\"make_calls\": %llu, \"c_make\": %.3f}\n",
           pos.size(), depth, (unsigned long long)leaves,
           (unsigned long long)n_count, (double)ops_count / n_count,
           (unsigned long long)n_gen, (double)ops_gen / n_gen, (double)gen_moves_total / n_gen,
           (unsigned long long)n_make, (double)ops_make / n_make);
    return 0;
}
