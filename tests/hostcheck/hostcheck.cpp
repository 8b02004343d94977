// Test-only: the product's move generator (perft_gpu_b200/csrc/movegen.cuh)
// compiled for the host, so the CPU test suite can check it against the
// oracle without a GPU.  Not part of the product library.
#include <stdint.h>
#include <string.h>

#include "../../perft_gpu_b200/csrc/movegen.cuh"

namespace pg {
void build_tables();
}

using namespace pg;

namespace {
struct VecSink {
    u32 *out;
    u32 n;
    void operator()(u32 m) { out[n++] = m; }
};

template <int SV>
uint64_t perft_rel(const Board &b, uint32_t depth)
{
    if (depth == 0) return 1;
    if (depth == 1) return count_moves<SV>(b);
    u32 moves[256];
    VecSink s{moves, 0};
    gen_moves<SV>(b, s);
    uint64_t total = 0;
    for (u32 i = 0; i < s.n; i++) total += perft_rel<SV>(make_child(b, moves[i]), depth - 1);
    return total;
}
}  // namespace

// Calls f.template operator()<SV>() for the runtime variant sv (0..4).
template <class F>
auto with_sv(int sv, F f)
{
    switch (sv) {
    case SV_MAGIC: return f.template operator()<SV_MAGIC>();
    case SV_KOGGE_FMA: return f.template operator()<SV_KOGGE_FMA>();
    case SV_KOGGE_SPLIT: return f.template operator()<SV_KOGGE_SPLIT>();
    case SV_HYBRID: return f.template operator()<SV_HYBRID>();
    default: return f.template operator()<SV_KOGGE>();
    }
}

extern "C" {

int hc_init(void)
{
    build_tables();
    return 0;
}

uint32_t hc_count(const uint64_t pos[6], int sv)
{
    const Board b = from_pos48(pos);
    return with_sv(sv, [&]<int SV>() { return count_moves<SV>(b); });
}

// Children of pos as pos48 boards; returns the number of moves.
uint32_t hc_children(const uint64_t pos[6], int sv, uint64_t *out)
{
    const Board b = from_pos48(pos);
    u32 moves[256];
    VecSink s{moves, 0};
    with_sv(sv, [&]<int SV>() { gen_moves<SV>(b, s); return 0; });
    for (u32 i = 0; i < s.n; i++) {
        Board c = make_child(b, moves[i]);
        to_pos48(c, out + 6 * i);
    }
    return s.n;
}

// Children as the tile kernel makes them: moves carrying the mover's planes
// (gen_moves<SV, true>), children made without piece lookups
// (make_child<true>), with a parent slot in bits 16-23 as the kernel's items
// have.  Also writes the 16-bit moves to mv16.
uint32_t hc_children_mover(const uint64_t pos[6], int sv, uint64_t *out, uint16_t *mv16)
{
    const Board b = from_pos48(pos);
    u32 moves[256];
    VecSink s{moves, 0};
    with_sv(sv, [&]<int SV>() { gen_moves<SV, true>(b, s); return 0; });
    for (u32 i = 0; i < s.n; i++) {
        Board c = make_child<true>(b, moves[i] | (0xA5u << 16));
        to_pos48(c, out + 6 * i);
        mv16[i] = (uint16_t)moves[i];
    }
    return s.n;
}

// Children made from the mirrored parent (make_child_mirrored), as the tile
// kernel makes them; the caller compares them with hc_children.
uint32_t hc_children_mirrored(const uint64_t pos[6], uint64_t *out)
{
    const Board b = from_pos48(pos);
    u32 moves[256];
    VecSink s{moves, 0};
    gen_moves<SV_KOGGE>(b, s);
    const Board f = flip_board(b);
    for (u32 i = 0; i < s.n; i++) to_pos48(make_child_mirrored(f, moves[i] | (0x5Au << 16)), out + 6 * i);
    return s.n;
}

// Move counts of the children made from the mirrored parent with the king
// squares handed to the count (as the tile kernel does), next to the plain
// count of the same children; returns the number of mismatches.
uint32_t hc_counts_known_kings(const uint64_t pos[6], int sv)
{
    const Board b = from_pos48(pos);
    u32 moves[256];
    VecSink s{moves, 0};
    gen_moves<SV_KOGGE>(b, s);
    const Board f = flip_board(b);
    const int oKing = ctz(f.kings & ~f.mine), sKing = ctz(f.kings & f.mine);
    uint32_t bad = 0;
    for (u32 i = 0; i < s.n; i++) {
        int tk = -1;
        u64 occ = 0, theirs = 0;
        const Board c = make_child_mirrored(f, moves[i], &tk, sKing, &occ, &theirs);
        const uint32_t want = with_sv(sv, [&]<int SV>() { return count_moves<SV>(c); });
        const uint32_t got = with_sv(sv, [&]<int SV>() {
            return SvTraits<SV>::kogge ? count_moves_fused<SV>(c, oKing, tk) : count_moves<SV>(c);
        });
        const uint32_t got2 = with_sv(sv, [&]<int SV>() { return count_moves_ko<SV>(c, oKing, tk, occ, theirs); });
        bad += (got != want) + (got2 != want);
    }
    return bad;
}

uint64_t hc_perft(const uint64_t pos[6], uint32_t depth, int sv)
{
    const Board b = from_pos48(pos);
    return with_sv(sv, [&]<int SV>() { return perft_rel<SV>(b, depth); });
}

void hc_roundtrip(const uint64_t pos[6], uint64_t out[6])
{
    to_pos48(from_pos48(pos), out);
}
}
