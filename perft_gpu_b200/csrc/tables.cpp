// Host construction of the lookup tables used by the move generator:
// king/knight attacks, empty-board slider rays, between/line masks
// (the reference builds the same sets in MoveGeneratorBitboard.h:982-1031),
// and fancy-magic slider tables.
//
// The magic multipliers are found here by a seeded random search (the
// published trial-and-error method: sparse random candidates, rejected on a
// destructive index collision).  No third-party magic constants are used;
// the search is deterministic, so every process builds identical tables.
#include <string.h>

#include <mutex>

#include "movegen.cuh"

namespace pg {

Tables h_tables;
u64 h_magic[MAGIC_TABLE_ENTRIES];

namespace {

u64 ray_walk(int sq, int df, int dr, u64 occ, bool stopAtEdgeExclusive)
{
    u64 m = 0;
    int f = (sq & 7) + df, r = (sq >> 3) + dr;
    while (f >= 0 && f < 8 && r >= 0 && r < 8) {
        int nf = f + df, nr = r + dr;
        bool last = !(nf >= 0 && nf < 8 && nr >= 0 && nr < 8);
        if (stopAtEdgeExclusive && last) break;
        u64 bit = 1ULL << (r * 8 + f);
        m |= bit;
        if (occ & bit) break;
        f = nf;
        r = nr;
    }
    return m;
}

const int ROOK_DIRS[4][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}};
const int BISHOP_DIRS[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

u64 slow_attacks(int sq, u64 occ, const int dirs[4][2])
{
    u64 a = 0;
    for (int d = 0; d < 4; d++) a |= ray_walk(sq, dirs[d][0], dirs[d][1], occ, false);
    return a;
}

u64 relevant_mask(int sq, const int dirs[4][2])
{
    u64 m = 0;
    for (int d = 0; d < 4; d++) m |= ray_walk(sq, dirs[d][0], dirs[d][1], 0, true);
    return m;
}

struct Rng {
    u64 s;
    u64 next()
    {
        // xorshift64*
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return s * 0x2545F4914F6CDD1DULL;
    }
    u64 sparse() { return next() & next() & next(); }
};

// Finds a multiplier mapping every occupancy subset of mask to a table slot
// of 2^bits entries without destructive collisions; fills table[0..2^bits).
u64 find_magic(int sq, u64 mask, const int dirs[4][2], u64 *table, Rng &rng)
{
    const int bits = popc(mask);
    const int n = 1 << bits;
    static u64 occs[4096], atts[4096], used[4096];
    static u32 epoch[4096];
    static u32 cur = 0;
    int k = 0;
    u64 sub = 0;
    do {
        occs[k] = sub;
        atts[k] = slow_attacks(sq, sub, dirs);
        k++;
        sub = (sub - mask) & mask;
    } while (sub);
    for (;;) {
        u64 magic = rng.sparse();
        if (popc((mask * magic) & 0xFF00000000000000ULL) < 6) continue;
        cur++;
        bool ok = true;
        for (int i = 0; i < n && ok; i++) {
            u32 idx = (u32)((occs[i] * magic) >> (64 - bits));
            if (epoch[idx] != cur) {
                epoch[idx] = cur;
                used[idx] = atts[i];
            } else if (used[idx] != atts[i]) {
                ok = false;
            }
        }
        if (!ok) continue;
        for (int i = 0; i < n; i++) table[i] = 0;
        for (int i = 0; i < n; i++) table[(occs[i] * magic) >> (64 - bits)] = atts[i];
        return magic;
    }
}

std::once_flag g_builtOnce;

void build_tables_once()
{
    Tables &t = h_tables;
    memset(&t, 0, sizeof(t));
    for (int s = 0; s < 64; s++) {
        const u64 b = 1ULL << s;
        t.king[s] = sh_n(b) | sh_s(b) | sh_e(b) | sh_w(b) | sh_ne(b) | sh_nw(b) | sh_se(b) | sh_sw(b);
        t.pawnUp[s] = pawn_att_up(b);
        t.bit[s] = b;
        // rights of the side to move: 1 king side (rook h1), 2 queen side (a1);
        // of the opponent: 4 king side (h8), 8 queen side (a8)
        t.castleClear[s] = (uint8_t)(s == 7 ? 1 : s == 0 ? 2 : s == 63 ? 4 : s == 56 ? 8 : 0);
        t.knight[s] = knight_set_att(b);
        t.rookRays[s] = slow_attacks(s, 0, ROOK_DIRS);
        t.bishopRays[s] = slow_attacks(s, 0, BISHOP_DIRS);
    }
    for (int a = 0; a < 64; a++) {
        for (int b = 0; b < 64; b++) {
            if (a == b) continue;
            const int dirsAll[8][2] = {{0, 1}, {0, -1}, {1, 0}, {-1, 0}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
            for (int d = 0; d < 8; d++) {
                u64 ray = ray_walk(a, dirsAll[d][0], dirsAll[d][1], 0, false);
                if (!(ray & (1ULL << b))) continue;
                // squares from a towards b, stopping before b
                t.between[a][b] = ray_walk(a, dirsAll[d][0], dirsAll[d][1], 1ULL << b, false) & ~(1ULL << b);
                t.pairInfo[a][b] = (uint8_t)(popc(t.between[a][b]) | ((dirsAll[d][0] && dirsAll[d][1]) ? 8 : 0));
                u64 back = ray_walk(a, -dirsAll[d][0], -dirsAll[d][1], 0, false);
                t.line[a][b] = ray | back | (1ULL << a);
            }
        }
    }
    Rng rng{0x9E3779B97F4A7C15ULL};
    u32 off = 0;
    for (int s = 0; s < 64; s++) {
        u64 mask = relevant_mask(s, ROOK_DIRS);
        t.rookMask[s] = mask;
        t.rookShift[s] = 64 - popc(mask);
        t.rookOffset[s] = off;
        t.rookMagic[s] = find_magic(s, mask, ROOK_DIRS, &h_magic[off], rng);
        off += 1u << popc(mask);
    }
    for (int s = 0; s < 64; s++) {
        u64 mask = relevant_mask(s, BISHOP_DIRS);
        t.bishopMask[s] = mask;
        t.bishopShift[s] = 64 - popc(mask);
        t.bishopOffset[s] = off;
        t.bishopMagic[s] = find_magic(s, mask, BISHOP_DIRS, &h_magic[off], rng);
        off += 1u << popc(mask);
    }
}

}  // namespace

// Builds the tables once per process.  Every caller (engine start-up, the
// allocation-free entry point, the host-side entry points, on any thread)
// returns only after the tables are complete: std::call_once blocks
// concurrent callers until the first one has finished filling them.
void build_tables()
{
    std::call_once(g_builtOnce, build_tables_once);
}

}  // namespace pg
