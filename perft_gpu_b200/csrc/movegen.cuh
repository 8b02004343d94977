// Side-relative bitboard move generator shared by the CUDA kernels and the
// host utilities (FEN / UCI move parsing, position generators).
//
// Semantics follow the reference move generator (ankan-ban/perft_gpu,
// MoveGeneratorBitboard.h): legal-move counting without generation
// (countMoves :3008-3295, out of check :2828-3002), generation
// (generateMoves :2471-2823, out of check :2269-2465) and make-move
// (makeMove :3310-3570 with exact en-passant flagging, switches.h:48).
//
// Representation differs from the reference on purpose: every board is kept
// from the point of view of the side to move ("mine" moves up the board).
// A black-to-move position is stored vertically mirrored with colours
// swapped.  Perft is invariant under that mirror, so counts are identical,
// and the kernels need no per-side templates or side-dependent branches:
// a warp whose lanes hold positions of different sides runs one code path.
//
// Board: six 64-bit planes, 48 bytes (same size and plane order as the
// reference's HexaBitBoardPosition, chess.h:208-230, with "white pieces"
// replaced by "pieces of the side to move"):
//   mine, pawns, knights, bq (bishops|queens), rq (rooks|queens), kings
// Pawns never stand on ranks 1/8, so the pawn plane carries the state:
//   bits 0-1  castling rights of the side to move (1 king side, 2 queen side)
//   bits 2-3  castling rights of the opponent
//   bits 4-7  en-passant file + 1 (target on relative rank 6), 0 if none
//   bit 63    1 when the real side to move is black
// For a white-to-move position bits 0-7 coincide with the reference's packed
// state byte.
//
// Moves are 16 bit: from (0-5), to (6-11), flags (12-15) with the
// reference's CMove codes (chess.h:269-293).  Squares are relative.
#pragma once

#include <stdint.h>

// Build-time alternatives, each kept for A/B measurement; the defaults are
// the measured-fastest choices on B200.
// PG_FUSED_COUNT 1: Kogge-Stone counts use count_moves_fused.
#ifndef PG_FUSED_COUNT
#define PG_FUSED_COUNT 1
#endif
// PG_RANK_SUB 1: east/west rays of the fused count by carry subtraction.
#ifndef PG_RANK_SUB
#define PG_RANK_SUB 1
#endif
// PG_KNIGHT_LUT: knight moves of the Kogge-Stone variants; 0 = eight jump
// shifts over the whole knight set, 1 = one table lookup per knight.
#ifndef PG_KNIGHT_LUT
#define PG_KNIGHT_LUT 1
#endif
// PG_COUNT_TABLES 1: the fused count takes a king's pawn checkers and each
// pin line's length and kind from tables instead of computing them.
#ifndef PG_COUNT_TABLES
#define PG_COUNT_TABLES 1
#endif
// PG_MAKE_TABLES 1: make-move takes the from/to bits and the castling rights
// a move clears from tables, and tests the moving piece against the from bit.
#ifndef PG_MAKE_TABLES
#define PG_MAKE_TABLES 1
#endif
// PG_KS_LINE 1: the fused count fills both directions of a line from one
// propagator chain.
#ifndef PG_KS_LINE
#define PG_KS_LINE 1
#endif
// PG_CTZ32 1: bit scans of 64-bit words as two 32-bit scans.
#ifndef PG_CTZ32
#define PG_CTZ32 1
#endif
// PG_GEN_MAGIC 1: move generation looks up each slider's targets in the
// magic tables whatever the slider variant.
#ifndef PG_GEN_MAGIC
#define PG_GEN_MAGIC 1
#endif
// PG_MOVER_BITS 1: the tile kernel's generated items carry the moving
// piece's planes, so its make-move needs no piece lookups.  Measured 0.7%
// slower on the 4096-position batch (the lookups were cheaper than the
// extra live state), so off by default.
#ifndef PG_MOVER_BITS
#define PG_MOVER_BITS 0
#endif
// PG_GEN_MAGIC_ATTACKS 1: generation also builds the opponent's attack map
// from magic lookups, one per opponent slider.
#ifndef PG_GEN_MAGIC_ATTACKS
#define PG_GEN_MAGIC_ATTACKS 1
#endif

#ifdef __CUDACC__
#define PG_HD __host__ __device__ __forceinline__
#else
#define PG_HD inline
#endif

namespace pg {

typedef uint64_t u64;
typedef uint32_t u32;

struct Board {
    u64 mine, pawns, knights, bq, rq, kings;
};

enum : u64 {
    RANKS2TO7 = 0x00FFFFFFFFFFFF00ULL,
    RANK1 = 0x00000000000000FFULL,
    RANK3 = 0x0000000000FF0000ULL,
    RANK5 = 0x000000FF00000000ULL,
    RANK8 = 0xFF00000000000000ULL,
    FILEA = 0x0101010101010101ULL,
    FILEB = 0x0202020202020202ULL,
    FILEG = 0x4040404040404040ULL,
    FILEH = 0x8080808080808080ULL,
    SIDE_BIT = 0x8000000000000000ULL,
};

enum : u32 {
    MF_QUIET = 0,
    MF_DOUBLE_PUSH = 1,
    MF_KING_CASTLE = 2,
    MF_QUEEN_CASTLE = 3,
    MF_CAPTURE = 4,
    MF_EP = 5,
    MF_PROMO = 8,  // | 0 knight, 1 bishop, 2 rook, 3 queen; | 4 capture
};

// Slider attack implementation used by a kernel instantiation.
enum SliderVariant : int {
    SV_KOGGE = 0,      // occluded fills, all pieces of a set at once, no tables
    SV_MAGIC = 1,      // fancy magic lookups, one per piece
    SV_KOGGE_FMA = 2,  // occluded fills with every constant shift on the FMA pipe
    SV_KOGGE_SPLIT = 3,  // left shifts split: high word on the ALU, low word on the FMA pipe
    SV_HYBRID = 4,       // opponent attack map by split-shift fills, own slider moves by magic lookups
    SV_COUNT = 5,
};

// How a Kogge-Stone fill issues its constant shifts.
enum ShiftMode : int { SH_ALU = 0, SH_FMA = 1, SH_SPLIT = 2 };

// Compile-time properties of a variant.
template <int SV>
struct SvTraits {
    static constexpr bool kogge = SV != SV_MAGIC;
    static constexpr bool ownMagic = SV == SV_HYBRID;  // own slider moves by lookups
    static constexpr int shift =
        SV == SV_KOGGE_FMA ? SH_FMA : ((SV == SV_KOGGE_SPLIT || SV == SV_HYBRID) ? SH_SPLIT : SH_ALU);
};

// ------------------------------------------------------------------ tables
// Built once on the host (tables.cpp) and copied to a __device__ symbol.
struct Tables {
    u64 king[64];
    u64 knight[64];
    u64 rookRays[64];    // empty-board rook attacks
    u64 bishopRays[64];  // empty-board bishop attacks
    u64 between[64][64]; // squares strictly between two squares on a line
    u64 line[64][64];    // full line through two squares
    u64 rookMask[64], bishopMask[64];
    u64 rookMagic[64], bishopMagic[64];
    u32 rookOffset[64], bishopOffset[64];
    u32 rookShift[64], bishopShift[64];
    u64 pawnUp[64];         // squares a side-to-move pawn on s attacks (its checkers of a king on s)
    uint8_t pairInfo[64][64];  // squares strictly between (bits 0-2) and 8 when the line is a diagonal
    u64 bit[64];               // 1 << s
    uint8_t castleClear[64];   // castling rights lost when a piece leaves or lands on s (rook corners)
};

// Total entries of the fancy-magic attack table (rook part then bishop part).
constexpr u32 MAGIC_TABLE_ENTRIES = 102400 + 5248;

extern Tables h_tables;
extern u64 h_magic[MAGIC_TABLE_ENTRIES];

#ifdef __CUDACC__
// The one CUDA translation unit (engine.cu) defines the device copies.
__device__ Tables d_tables;
__device__ u64 d_magic[MAGIC_TABLE_ENTRIES];
// c_pow2[k] = 2^k, uploaded at start-up.  Shift amounts read from here are
// opaque to the compiler, so a multiply by them stays an integer
// multiply-add on the FMA pipe instead of being folded back into a shift on
// the (busier) ALU pipe.
__constant__ u32 c_pow2[32];
#endif

#ifdef __CUDA_ARCH__
#define PG_TAB(field) (__ldg(&d_tables.field))
#define PG_MAGIC(i) (__ldg(&d_magic[(i)]))
#else
#define PG_TAB(field) (h_tables.field)
#define PG_MAGIC(i) (h_magic[(i)])
#endif

// ------------------------------------------------------------- bit helpers
PG_HD int popc(u64 x)
{
#ifdef __CUDA_ARCH__
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}

// Popcount of the high byte (the eighth rank) and of the low word (ranks 1-4).
PG_HD int popc_byte7(u64 x)
{
#ifdef __CUDA_ARCH__
    return __popc((u32)(x >> 56));
#else
    return __builtin_popcount((unsigned)(x >> 56));
#endif
}
PG_HD int popc_lo(u64 x)
{
#ifdef __CUDA_ARCH__
    return __popc((u32)x);
#else
    return __builtin_popcount((unsigned)x);
#endif
}

PG_HD int ctz(u64 x)
{
#ifdef __CUDA_ARCH__
#if PG_CTZ32
    // two 32-bit scans and a select
    const u32 lo = (u32)x;
    return lo ? __ffs(lo) - 1 : __ffs((u32)(x >> 32)) + 31;
#else
    return __ffsll((long long)x) - 1;
#endif
#else
    return __builtin_ctzll(x);
#endif
}

// Calls f(square) for every set bit in ascending order; on the device the
// two 32-bit halves are walked separately (32-bit bit scans and clears).
template <class F>
PG_HD void for_each_bit(u64 x, F f)
{
#ifdef __CUDA_ARCH__
    for (u32 w = (u32)x; w; w &= w - 1) f(__ffs(w) - 1);
    for (u32 w = (u32)(x >> 32); w; w &= w - 1) f(__ffs(w) + 31);
#else
    while (x) {
        f(ctz(x));
        x &= x - 1;
    }
#endif
}

// Vertical mirror (rank r -> 7 - r): a byte swap.
PG_HD u64 flipv(u64 x)
{
#ifdef __CUDA_ARCH__
    u32 lo = (u32)x, hi = (u32)(x >> 32);
    u32 nlo = __byte_perm(hi, 0, 0x0123);
    u32 nhi = __byte_perm(lo, 0, 0x0123);
    return ((u64)nhi << 32) | nlo;
#else
    return __builtin_bswap64(x);
#endif
}

PG_HD u64 maskIf(bool c) { return (u64)0 - (u64)c; }

// ------------------------------------------------------- one-square shifts
PG_HD u64 sh_n(u64 x) { return x << 8; }
PG_HD u64 sh_s(u64 x) { return x >> 8; }
PG_HD u64 sh_e(u64 x) { return (x << 1) & ~FILEA; }
PG_HD u64 sh_w(u64 x) { return (x >> 1) & ~FILEH; }
PG_HD u64 sh_ne(u64 x) { return (x << 9) & ~FILEA; }
PG_HD u64 sh_nw(u64 x) { return (x << 7) & ~FILEH; }
PG_HD u64 sh_se(u64 x) { return (x >> 7) & ~FILEA; }
PG_HD u64 sh_sw(u64 x) { return (x >> 9) & ~FILEH; }

// ------------------------------------------------- FMA-pipe constant shifts
// 64-bit shifts by a constant K written as 32x32 multiplies by 2^K, so they
// issue on the FMA pipe (IMAD.WIDE / IMAD / IMAD.HI) rather than the ALU.
// Left:  t = lo * 2^K (wide) gives lo << K and lo >> (32-K); hi' = hi*2^K + that.
// Right: hi * 2^(32-K) (wide) plus umulhi(lo, 2^(32-K)) = lo >> K gives both
// words at once (the two parts occupy disjoint bits).  Host builds shift.
// n + popc(x).  With PG_POPC_IMAD the two half-word counts are added by
// multiply-adds with the opaque factor c_pow2[0] = 1: the FMA pipe, which the
// count leaves mostly idle, instead of an IADD3 on the ALU pipe that binds it.
#ifndef PG_POPC_IMAD
#define PG_POPC_IMAD 1
#endif
PG_HD u32 add_popc(u32 n, u64 x)
{
#if defined(__CUDA_ARCH__) && PG_POPC_IMAD
    const u32 one = c_pow2[0];
    return (u32)__popc((u32)(x >> 32)) * one + ((u32)__popc((u32)x) * one + n);
#else
    return n + popc(x);
#endif
}

template <int K>
PG_HD u64 shl_fma(u64 x)
{
#ifdef __CUDA_ARCH__
    const u32 lo = (u32)x, hi = (u32)(x >> 32);
    if (K == 0) return x;
    if (K >= 32) {
        if (K == 32) return (u64)lo << 32;
        return (u64)(lo * c_pow2[K - 32]) << 32;
    }
    const u32 m = c_pow2[K];
    const u64 t = (u64)lo * m;
    const u32 nhi = hi * m + (u32)(t >> 32);
    return ((u64)nhi << 32) | (u32)t;
#else
    return x << K;
#endif
}

template <int K>
PG_HD u64 shr_fma(u64 x)
{
#ifdef __CUDA_ARCH__
    const u32 lo = (u32)x, hi = (u32)(x >> 32);
    if (K == 0) return x;
    if (K >= 32) {
        if (K == 32) return hi;
        return __umulhi(hi, c_pow2[64 - K]);
    }
    const u32 m = c_pow2[32 - K];
    return (u64)hi * m + __umulhi(lo, m);
#else
    return x >> K;
#endif
}

// Left shift with the high word from an ALU funnel shift and the low word
// from an integer multiply (FMA pipe): one instruction on each pipe.
template <int K>
PG_HD u64 shl_split(u64 x)
{
#ifdef __CUDA_ARCH__
    const u32 lo = (u32)x, hi = (u32)(x >> 32);
    if (K == 0) return x;
    if (K >= 32) return shl_fma<K>(x);
    const u32 nhi = __funnelshift_l(lo, hi, K);
    const u32 nlo = lo * c_pow2[K];
    return ((u64)nhi << 32) | nlo;
#else
    return x << K;
#endif
}

template <int K, int MODE>
PG_HD u64 shl(u64 x)
{
    if (MODE == SH_FMA) return shl_fma<K>(x);
    if (MODE == SH_SPLIT) return shl_split<K>(x);
    return x << K;
}
template <int K, int MODE>
PG_HD u64 shr(u64 x)
{
    if (MODE == SH_FMA) return shr_fma<K>(x);
    return x >> K;
}

// ------------------------------------------------------------ Kogge-Stone
// Occluded fill of generator set g through propagator p, then one more step:
// every square attacked in that direction (first blocker included).  The
// fill is OR-distributive over generators, and same-direction rays of
// different pieces never share a non-own square, so per-direction popcounts
// of a whole piece set sum to the per-piece move counts.
template <int S, bool LEFT, int FMA>
PG_HD u64 ks_dir(u64 g, u64 p, u64 wrap)
{
    p &= wrap;
    if (LEFT) {
        g |= p & shl<S, FMA>(g);
        p &= shl<S, FMA>(p);
        g |= p & shl<2 * S, FMA>(g);
        p &= shl<2 * S, FMA>(p);
        g |= p & shl<4 * S, FMA>(g);
        return shl<S, FMA>(g) & wrap;
    } else {
        g |= p & shr<S, FMA>(g);
        p &= shr<S, FMA>(p);
        g |= p & shr<2 * S, FMA>(g);
        p &= shr<2 * S, FMA>(p);
        g |= p & shr<4 * S, FMA>(g);
        return shr<S, FMA>(g) & wrap;
    }
}

template <int F = SH_ALU> PG_HD u64 ks_north(u64 g, u64 p) { return ks_dir<8, true, F>(g, p, ~0ULL); }
template <int F = SH_ALU> PG_HD u64 ks_south(u64 g, u64 p) { return ks_dir<8, false, F>(g, p, ~0ULL); }
template <int F = SH_ALU> PG_HD u64 ks_east(u64 g, u64 p) { return ks_dir<1, true, F>(g, p, ~FILEA); }
template <int F = SH_ALU> PG_HD u64 ks_west(u64 g, u64 p) { return ks_dir<1, false, F>(g, p, ~FILEH); }
template <int F = SH_ALU> PG_HD u64 ks_ne(u64 g, u64 p) { return ks_dir<9, true, F>(g, p, ~FILEA); }
template <int F = SH_ALU> PG_HD u64 ks_nw(u64 g, u64 p) { return ks_dir<7, true, F>(g, p, ~FILEH); }
template <int F = SH_ALU> PG_HD u64 ks_se(u64 g, u64 p) { return ks_dir<7, false, F>(g, p, ~FILEA); }
template <int F = SH_ALU> PG_HD u64 ks_sw(u64 g, u64 p) { return ks_dir<9, false, F>(g, p, ~FILEH); }

template <int F = SH_ALU>
PG_HD u64 ks_diag(u64 g, u64 empty)
{
    return ks_ne<F>(g, empty) | ks_nw<F>(g, empty) | ks_se<F>(g, empty) | ks_sw<F>(g, empty);
}
template <int F = SH_ALU>
PG_HD u64 ks_orth(u64 g, u64 empty)
{
    return ks_north<F>(g, empty) | ks_south<F>(g, empty) | ks_east<F>(g, empty) | ks_west<F>(g, empty);
}

// Per-direction move counts of a whole slider set (targets = squares the
// pieces may land on).
template <int F = SH_ALU>
PG_HD int ks_count_diag(u64 g, u64 empty, u64 targets)
{
    return popc(ks_ne<F>(g, empty) & targets) + popc(ks_nw<F>(g, empty) & targets) +
           popc(ks_se<F>(g, empty) & targets) + popc(ks_sw<F>(g, empty) & targets);
}
template <int F = SH_ALU>
PG_HD int ks_count_orth(u64 g, u64 empty, u64 targets)
{
    return popc(ks_north<F>(g, empty) & targets) + popc(ks_south<F>(g, empty) & targets) +
           popc(ks_east<F>(g, empty) & targets) + popc(ks_west<F>(g, empty) & targets);
}

// ------------------------------------------------------------------ magics
PG_HD u64 magic_bishop(int sq, u64 occ)
{
    u64 idx = ((occ & PG_TAB(bishopMask[sq])) * PG_TAB(bishopMagic[sq])) >> PG_TAB(bishopShift[sq]);
    return PG_MAGIC(PG_TAB(bishopOffset[sq]) + (u32)idx);
}
PG_HD u64 magic_rook(int sq, u64 occ)
{
    u64 idx = ((occ & PG_TAB(rookMask[sq])) * PG_TAB(rookMagic[sq])) >> PG_TAB(rookShift[sq]);
    return PG_MAGIC(PG_TAB(rookOffset[sq]) + (u32)idx);
}

// Attacks of the piece on square sq given occupancy occ.
template <int SV>
PG_HD u64 bishop_att(int sq, u64 occ)
{
    if (SV == SV_MAGIC) return magic_bishop(sq, occ);
    return ks_diag<SvTraits<SV>::shift>(1ULL << sq, ~occ);
}
template <int SV>
PG_HD u64 rook_att(int sq, u64 occ)
{
    if (SV == SV_MAGIC) return magic_rook(sq, occ);
    return ks_orth<SvTraits<SV>::shift>(1ULL << sq, ~occ);
}

// Union of the attacks of a slider set; occ excludes transparent squares.
template <int SV>
PG_HD u64 bishop_set_att(u64 set, u64 occ)
{
    if (SvTraits<SV>::kogge) return ks_diag<SvTraits<SV>::shift>(set, ~occ);
    u64 a = 0;
    for_each_bit(set, [&](int sq) { a |= magic_bishop(sq, occ); });
    return a;
}
template <int SV>
PG_HD u64 rook_set_att(u64 set, u64 occ)
{
    if (SvTraits<SV>::kogge) return ks_orth<SvTraits<SV>::shift>(set, ~occ);
    u64 a = 0;
    for_each_bit(set, [&](int sq) { a |= magic_rook(sq, occ); });
    return a;
}

// ------------------------------------------------------------ leaper sets
PG_HD u64 knight_set_att(u64 n)
{
    u64 l1 = (n >> 1) & 0x7f7f7f7f7f7f7f7fULL;
    u64 l2 = (n >> 2) & 0x3f3f3f3f3f3f3f3fULL;
    u64 r1 = (n << 1) & 0xfefefefefefefefeULL;
    u64 r2 = (n << 2) & 0xfcfcfcfcfcfcfcfcULL;
    u64 h1 = l1 | r1, h2 = l2 | r2;
    return (h1 << 16) | (h1 >> 16) | (h2 << 8) | (h2 >> 8);
}

// Knight move count of a knight set by the eight (injective) jump shifts.
PG_HD int knight_set_count(u64 n, u64 targets)
{
    const u64 notA = ~FILEA, notH = ~FILEH, notAB = ~(FILEA | FILEB), notGH = ~(FILEG | FILEH);
    return popc((n << 17) & notA & targets) + popc((n << 15) & notH & targets) +
           popc((n << 10) & notAB & targets) + popc((n << 6) & notGH & targets) +
           popc((n >> 6) & notAB & targets) + popc((n >> 10) & notGH & targets) +
           popc((n >> 15) & notA & targets) + popc((n >> 17) & notH & targets);
}

// Pawns of the side to move attack up, the opponent's attack down.
PG_HD u64 pawn_att_up(u64 p) { return sh_ne(p) | sh_nw(p); }
PG_HD u64 pawn_att_down(u64 p) { return sh_se(p) | sh_sw(p); }

// ---------------------------------------------------------- position setup
struct Ctx {
    u64 pawns, occ, mine, theirs, empty;
    u64 myK, tP, tN, tB, tR, tK;
    u64 attacked;  // squares attacked by the opponent (own king transparent)
    u32 st;        // state byte
    int ksq;
};

template <int SV>
PG_HD void setup_ctx(const Board &b, Ctx &c)
{
    c.pawns = b.pawns & RANKS2TO7;
    c.occ = c.pawns | b.knights | b.bq | b.rq | b.kings;
    c.mine = b.mine;
    c.theirs = c.occ ^ b.mine;
    c.empty = ~c.occ;
    c.myK = b.kings & b.mine;
    c.ksq = ctz(c.myK);
    c.tP = c.pawns & c.theirs;
    c.tN = b.knights & c.theirs;
    c.tB = b.bq & c.theirs;
    c.tR = b.rq & c.theirs;
    c.tK = b.kings & c.theirs;
    c.st = (u32)(b.pawns & 0xFF);
    const u64 occNoK = c.occ ^ c.myK;
    c.attacked = pawn_att_down(c.tP) | knight_set_att(c.tN) | PG_TAB(king[ctz(c.tK)]) |
                 bishop_set_att<SV>(c.tB, occNoK) | rook_set_att<SV>(c.tR, occNoK);
}

// Pinned pieces of the side to move (findPinnedPieces, MoveGeneratorBitboard.h:1213-1249).
PG_HD u64 pinned_of(const Ctx &c)
{
    u64 pinned = 0;
    for_each_bit((PG_TAB(rookRays[c.ksq]) & c.tR) | (PG_TAB(bishopRays[c.ksq]) & c.tB), [&](int s) {
        const u64 blk = PG_TAB(between[c.ksq][s]) & c.occ;
        if (blk && !(blk & (blk - 1))) pinned |= blk & c.mine;
    });
    return pinned;
}

// Horizontal discovered-check test for an en-passant capture by an unpinned
// pawn (MoveGeneratorBitboard.h:3079-3086): true when removing both pawns
// exposes the king to a rook/queen along the rank.
PG_HD bool ep_exposes_king(const Ctx &c, u64 src, u64 captured)
{
    if (!(c.myK & RANK5)) return false;
    u64 pro = c.empty | src | captured;
    return ((ks_east(c.myK, pro) | ks_west(c.myK, pro)) & c.tR) != 0;
}

// ------------------------------------------------------------------- count
// Check mask of the side to move: every square when not in check; the
// checker plus the squares between it and the king in single check; nothing
// in double check.  Non-king moves must land inside it.  A pinned piece can
// never resolve a check (its pin line meets the check line only at the
// king), so pinned moves are dropped in check.  This folds the reference's
// separate out-of-check routines (countMovesOutOfCheck /
// generateMovesOutOfCheck) into the main path, so a warp with one lane in
// check does not run a second move generator for it.
template <int SV>
PG_HD u64 check_mask(const Ctx &c)
{
    if (!(c.attacked & c.myK)) return ~0ULL;
    const u64 chk = (pawn_att_up(c.myK) & c.tP) | (PG_TAB(knight[c.ksq]) & c.tN) |
                    (magic_bishop(c.ksq, c.occ) & c.tB) | (magic_rook(c.ksq, c.occ) & c.tR);
    if (chk & (chk - 1)) return 0;
    return chk | PG_TAB(between[c.ksq][ctz(chk)]);
}

// One Kogge-Stone direction for two generator sets sharing one propagator
// chain (built from the empty squares): the opponent's sliders add to the
// attack map, this side's unpinned sliders add their move count.
template <int S, bool LEFT, int MODE>
PG_HD void ks_pair(u64 eGen, u64 oGen, u64 empty, u64 wrap, u64 targets, u64 &attacked, u32 &n)
{
    const u64 p0 = empty & wrap;
    u64 e = eGen, o = oGen;
    if (LEFT) {
        const u64 p1 = p0 & shl<S, MODE>(p0);
        const u64 p2 = p1 & shl<2 * S, MODE>(p1);
        e |= p0 & shl<S, MODE>(e);
        o |= p0 & shl<S, MODE>(o);
        e |= p1 & shl<2 * S, MODE>(e);
        o |= p1 & shl<2 * S, MODE>(o);
        e |= p2 & shl<4 * S, MODE>(e);
        o |= p2 & shl<4 * S, MODE>(o);
        attacked |= shl<S, MODE>(e) & wrap;
        n += popc(shl<S, MODE>(o) & wrap & targets);
    } else {
        const u64 p1 = p0 & shr<S, MODE>(p0);
        const u64 p2 = p1 & shr<2 * S, MODE>(p1);
        e |= p0 & shr<S, MODE>(e);
        o |= p0 & shr<S, MODE>(o);
        e |= p1 & shr<2 * S, MODE>(e);
        o |= p1 & shr<2 * S, MODE>(o);
        e |= p2 & shr<4 * S, MODE>(e);
        o |= p2 & shr<4 * S, MODE>(o);
        attacked |= shr<S, MODE>(e) & wrap;
        n += popc(shr<S, MODE>(o) & wrap & targets);
    }
}

// Both directions of one line (up by S and down by S) for the two generator
// sets, from one propagator chain: the down-direction propagators are the
// up-direction ones shifted down (P & P>>S == (P & P<<S) >> S, and the
// second doubling step shifts by 3S).  For diagonals, p0 excludes files a
// and h for both directions: a diagonal ray only enters the file it moves
// towards as its last square, which the final step adds, and never enters
// the other one without wrapping.  wrapUp / wrapDown mask the final step.
template <int S, int MODE>
PG_HD void ks_line(u64 eGen, u64 oGen, u64 p0, u64 wrapUp, u64 wrapDown, u64 targets, u64 &attacked, u32 &n)
{
    const u64 p1 = p0 & shl<S, MODE>(p0);
    const u64 p2 = p1 & shl<2 * S, MODE>(p1);
    {
        u64 e = eGen, o = oGen;
        e |= p0 & shl<S, MODE>(e);
        o |= p0 & shl<S, MODE>(o);
        e |= p1 & shl<2 * S, MODE>(e);
        o |= p1 & shl<2 * S, MODE>(o);
        e |= p2 & shl<4 * S, MODE>(e);
        o |= p2 & shl<4 * S, MODE>(o);
        attacked |= shl<S, MODE>(e) & wrapUp;
        n = add_popc(n, shl<S, MODE>(o) & wrapUp & targets);
    }
    {
        const u64 q1 = shr<S, MODE>(p1), q2 = shr<3 * S, MODE>(p2);
        u64 e = eGen, o = oGen;
        e |= p0 & shr<S, MODE>(e);
        o |= p0 & shr<S, MODE>(o);
        e |= q1 & shr<2 * S, MODE>(e);
        o |= q1 & shr<2 * S, MODE>(o);
        e |= q2 & shr<4 * S, MODE>(e);
        o |= q2 & shr<4 * S, MODE>(o);
        attacked |= shr<S, MODE>(e) & wrapDown;
        n = add_popc(n, shr<S, MODE>(o) & wrapDown & targets);
    }
}

// 64-bit bit reversal (file h <-> a, rank 8 <-> 1 mirrored together).
PG_HD u64 brev64(u64 x)
{
#ifdef __CUDA_ARCH__
    return __brevll(x);
#else
    x = ((x >> 1) & 0x5555555555555555ULL) | ((x & 0x5555555555555555ULL) << 1);
    x = ((x >> 2) & 0x3333333333333333ULL) | ((x & 0x3333333333333333ULL) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0FULL) | ((x & 0x0F0F0F0F0F0F0F0FULL) << 4);
    return __builtin_bswap64(x);
#endif
}

// East attacks of a slider set by carry subtraction.  `os` is the occupancy
// with a sentinel on every a-file square: subtracting 2g from it borrows
// through the empty squares east of each slider g and stops at (and clears)
// the first occupied square or the next rank's sentinel, so os ^ (os - 2G)
// marks exactly the squares each slider reaches, blocker included, plus
// sentinels that the a-file mask removes.  Borrow chains of different
// sliders never overlap: a chain stops at or before the next slider east
// on its rank, and each subtraction starts just east of its slider.
PG_HD u64 east_sub(u64 G, u64 os)
{
    return (os ^ (os - (G + G))) & ~FILEA;
}

// One rank direction pair: the opponent's fill feeds the attack map, this
// side's fill is counted.  WEST mirrors the board with bit reversal.
template <bool WEST>
PG_HD void rank_pair(u64 eGen, u64 oGen, u64 os, u64 targets, u64 &attacked, u32 &n)
{
    if (!WEST) {
        attacked |= east_sub(eGen, os);
        n = add_popc(n, east_sub(oGen, os) & targets);
    } else {
        attacked |= brev64(east_sub(brev64(eGen), os));
        n = add_popc(n, brev64(east_sub(brev64(oGen), os)) & targets);
    }
}

// countMoves for the Kogge-Stone variants, fused:
//  * checkers come first, straight from the king square (pawn, knight and
//    two slider lookups), so the check mask is known before any move count;
//  * the opponent's attack map treats this side's king as opaque, which lets
//    every direction build one propagator chain for both the opponent's
//    fill and this side's fill; the only square an opaque king hides is the
//    one behind it on a slider checker's line, which is added back (x-ray).
//
// ksqIn / tksqIn: the squares of this side's and the opponent's king when the
// caller knows them (the tile kernel does: they follow from the parent), or
// negative to find them here.
//
// With OCC, occIn / theirsIn are the board's occupancy and the opponent's
// pieces, which make-move already has.
template <int SV, bool OCC = false>
PG_HD u32 count_moves_fused(const Board &b, int ksqIn = -1, int tksqIn = -1, u64 occIn = 0, u64 theirsIn = 0)
{
    constexpr int M = SvTraits<SV>::shift;
    const u64 pawns = b.pawns & RANKS2TO7;
    const u64 occ = OCC ? occIn : (pawns | b.knights | b.bq | b.rq | b.kings);
    const u64 mine = b.mine, theirs = OCC ? theirsIn : occ ^ mine, empty = ~occ, notMine = ~mine;
    const u64 myK = b.kings & mine;
    const int ksq = ksqIn >= 0 ? ksqIn : ctz(myK);
    const u64 tP = pawns & theirs, tN = b.knights & theirs, tB = b.bq & theirs, tR = b.rq & theirs;
    const u32 st = (u32)(b.pawns & 0xFF);

    // pins and slider checks: every opponent slider on a line through the
    // king (a sniper) either checks (nothing between), pins (exactly one own
    // piece between) or neither; each pinned piece may only move along its
    // pin line
    u64 pinned = 0, slChk = 0;
    u32 nPinned = 0;
    const u64 bRays = PG_TAB(bishopRays[ksq]);
    for_each_bit((PG_TAB(rookRays[ksq]) & tR) | (bRays & tB), [&](int s) {
        const u64 btw = PG_TAB(between[ksq][s]);
        const u64 blk = btw & occ;
        if (!blk) {
            slChk |= 1ULL << s;
            return;
        }
        if ((blk & (blk - 1)) || !(blk & mine)) return;
        pinned |= blk;
        const u32 info = PG_COUNT_TABLES ? PG_TAB(pairInfo[ksq][s]) : 0u;
        const bool diag = PG_COUNT_TABLES ? (info & 8) != 0
                                          : (((ksq ^ s) & 7) != 0 && ((ksq ^ s) >> 3) != 0);  // neither file nor rank
        if (blk & (diag ? b.bq : b.rq)) {
            nPinned += PG_COUNT_TABLES ? (info & 7) : popc(btw);
        } else if (blk & pawns) {
            if (diag) {
                const u64 cap = pawn_att_up(blk) & (1ULL << s);
                nPinned += popc(cap) + 3 * popc(cap & RANK8);
            } else if (((ksq ^ s) & 7) == 0) {
                const u64 p1 = sh_n(blk) & empty;
                nPinned += popc(p1) + popc(sh_n(p1 & RANK3) & empty);
            }
        }
    });
    const u64 chk = ((PG_COUNT_TABLES ? PG_TAB(pawnUp[ksq]) : pawn_att_up(myK)) & tP) | (PG_TAB(knight[ksq]) & tN) |
                    slChk;
    u64 cm = ~0ULL, xray = 0;
    if (chk) {
        cm = (chk & (chk - 1)) ? 0 : (chk | PG_TAB(between[ksq][ctz(chk)]));
        u64 sl = slChk;
        while (sl) {
            const int c = ctz(sl);
            sl &= sl - 1;
            xray |= PG_TAB(line[ksq][c]) & ~PG_TAB(between[ksq][c]) & ~(1ULL << c);
        }
    }
    const bool inCheck = chk != 0;
    u32 n = inCheck ? 0 : nPinned;  // pinned pieces never resolve a check
    const u64 targets = notMine & cm;

    // sliders and the opponent's slider attacks, direction by direction
    const u64 B = b.bq & mine & ~pinned, R = b.rq & mine & ~pinned;
    u64 attacked = 0;
    if (SvTraits<SV>::ownMagic) {
        attacked = ks_orth<M>(tR, empty) | ks_diag<M>(tB, empty);
        u64 x = B;
        while (x) {
            n += popc(magic_bishop(ctz(x), occ) & targets);
            x &= x - 1;
        }
        x = R;
        while (x) {
            n += popc(magic_rook(ctz(x), occ) & targets);
            x &= x - 1;
        }
    } else {
#if PG_KS_LINE
        ks_line<8, M>(tR, R, empty, ~0ULL, ~0ULL, targets, attacked, n);
#else
        ks_pair<8, true, M>(tR, R, empty, ~0ULL, targets, attacked, n);
        ks_pair<8, false, M>(tR, R, empty, ~0ULL, targets, attacked, n);
#endif
        if (PG_RANK_SUB) {
            rank_pair<false>(tR, R, occ | FILEA, targets, attacked, n);
            rank_pair<true>(tR, R, brev64(occ) | FILEA, targets, attacked, n);
        } else {
            ks_pair<1, true, M>(tR, R, empty, ~FILEA, targets, attacked, n);
            ks_pair<1, false, M>(tR, R, empty, ~FILEH, targets, attacked, n);
        }
#if PG_KS_LINE
        const u64 inner = empty & ~(FILEA | FILEH);
        ks_line<9, M>(tB, B, inner, ~FILEA, ~FILEH, targets, attacked, n);  // north-east, south-west
        ks_line<7, M>(tB, B, inner, ~FILEH, ~FILEA, targets, attacked, n);  // north-west, south-east
#else
        ks_pair<9, true, M>(tB, B, empty, ~FILEA, targets, attacked, n);
        ks_pair<7, true, M>(tB, B, empty, ~FILEH, targets, attacked, n);
        ks_pair<7, false, M>(tB, B, empty, ~FILEA, targets, attacked, n);
        ks_pair<9, false, M>(tB, B, empty, ~FILEH, targets, attacked, n);
#endif
    }
    attacked |= pawn_att_down(tP) | knight_set_att(tN) | PG_TAB(king[tksqIn >= 0 ? tksqIn : ctz(b.kings & theirs)]);

    // king
    n = add_popc(n, PG_TAB(king[ksq]) & notMine & ~(attacked | xray));
    if (!cm) return n;  // double check: king moves only

    // castling (relative squares: king e1, rooks h1/a1), never out of check
    if (!inCheck) {
        if ((st & 1) && !((occ | attacked) & 0x60ULL)) n++;
        if ((st & 2) && !(occ & 0x0EULL) && !(attacked & 0x0CULL)) n++;
    }

    // free pawns, set-wise
    const u64 P = pawns & mine & ~pinned;
    const u64 p1 = sh_n(P) & empty;
    const u64 p1c = p1 & cm;
    n += popc_lo(sh_n(p1 & RANK3) & empty & cm);  // double pushes land on the fourth rank
    const u64 capT = theirs & cm;
    const u64 cl = sh_nw(P) & capT, cr = sh_ne(P) & capT;
    // pushes land on empty squares and captures on occupied ones, so the push
    // and left-capture sets are disjoint and share one popcount; promotions
    // (the eighth rank, the high byte) add three more moves each
    const u64 pl = p1c | cl;
    n = add_popc(add_popc(n, pl), cr) + 3 * (popc_byte7(pl) + popc_byte7(cr));

    // en passant: out of check, or capturing the checking pawn
    const u32 epf = st >> 4;
    if (epf) {
        const u64 target = 1ULL << (39 + epf);
        const u64 captured = sh_s(target);
        if (!inCheck || (captured & cm)) {
            u64 srcs = pawn_att_down(target) & pawns & mine;
            while (srcs) {
                const u64 sb = srcs & (0 - srcs);
                srcs ^= sb;
                if (sb & pinned) {
                    if (!inCheck && (PG_TAB(line[ctz(sb)][ksq]) & target)) n++;
                } else if (myK & RANK5) {
                    const u64 pro = empty | sb | captured;
                    if (!((ks_east(myK, pro) | ks_west(myK, pro)) & tR)) n++;
                } else {
                    n++;
                }
            }
        }
    }

    // knights
    const u64 N = b.knights & mine & ~pinned;
    if (PG_KNIGHT_LUT) {
        for_each_bit(N, [&](int sq) { n += popc(PG_TAB(knight[sq]) & targets); });  // a loop: keep the short IADD3 latency
    } else {
        n += knight_set_count(N, targets);
    }
    return n;
}

template <int SV>
PG_HD u32 count_moves(const Board &b);

// count_moves with the two king squares supplied (Kogge-Stone variants; the
// magic variant finds them itself).
template <int SV>
PG_HD u32 count_moves_k(const Board &b, int ksq, int tksq)
{
    if (SvTraits<SV>::kogge && PG_FUSED_COUNT) return count_moves_fused<SV>(b, ksq, tksq);
    return count_moves<SV>(b);
}

// count_moves_k with the occupancy and the opponent's pieces supplied too.
template <int SV>
PG_HD u32 count_moves_ko(const Board &b, int ksq, int tksq, u64 occ, u64 theirs)
{
    if (SvTraits<SV>::kogge && PG_FUSED_COUNT) return count_moves_fused<SV, true>(b, ksq, tksq, occ, theirs);
    return count_moves<SV>(b);
}

// Legal move count of the side to move (countMoves).
template <int SV>
PG_HD u32 count_moves(const Board &b)
{
#if PG_FUSED_COUNT
    if (SvTraits<SV>::kogge) return count_moves_fused<SV>(b);
#endif
    Ctx c;
    setup_ctx<SV>(b, c);
    const u64 notMine = ~c.mine;
    u32 n = popc(PG_TAB(king[c.ksq]) & notMine & ~c.attacked);
    const u64 cm = check_mask<SV>(c);
    if (!cm) return n;  // double check: king moves only
    const bool inCheck = cm != ~0ULL;
    const u64 targets = notMine & cm;

    // castling (relative squares: king e1, rooks h1/a1), never out of check
    if (!inCheck) {
        if ((c.st & 1) && !((c.occ | c.attacked) & 0x60ULL)) n++;
        if ((c.st & 2) && !(c.occ & 0x0EULL) && !(c.attacked & 0x0CULL)) n++;
    }

    // pins: each pinned piece may only move along its pin line
    u64 pinned = 0;
    u64 snipers = (PG_TAB(rookRays[c.ksq]) & c.tR) | (PG_TAB(bishopRays[c.ksq]) & c.tB);
    while (snipers) {
        const int s = ctz(snipers);
        snipers &= snipers - 1;
        const u64 btw = PG_TAB(between[c.ksq][s]);
        const u64 blk = btw & c.occ;
        if (!blk || (blk & (blk - 1)) || !(blk & c.mine)) continue;
        pinned |= blk;
        if (inCheck) continue;
        const bool diag = (PG_TAB(bishopRays[c.ksq]) >> s) & 1;
        if (blk & (diag ? b.bq : b.rq)) {
            n += popc(btw);  // every square between king and pinner, minus its own, plus the capture
        } else if (blk & c.pawns) {
            if (diag) {
                const u64 cap = pawn_att_up(blk) & (1ULL << s);
                n += popc(cap) + 3 * popc(cap & RANK8);
            } else if (((c.ksq ^ s) & 7) == 0) {
                const u64 p1 = sh_n(blk) & c.empty;
                n += popc(p1) + popc(sh_n(p1 & RANK3) & c.empty);
            }
        }
    }

    // free pawns, set-wise
    const u64 P = c.pawns & c.mine & ~pinned;
    const u64 p1 = sh_n(P) & c.empty;
    const u64 p1c = p1 & cm;
    n += popc(p1c) + 3 * popc(p1c & RANK8);
    n += popc(sh_n(p1 & RANK3) & c.empty & cm);
    const u64 capT = c.theirs & cm;
    const u64 cl = sh_nw(P) & capT, cr = sh_ne(P) & capT;
    n += popc(cl) + popc(cr) + 3 * (popc(cl & RANK8) + popc(cr & RANK8));

    // en passant: out of check, or capturing the checking pawn
    const u32 epf = c.st >> 4;
    if (epf) {
        const u64 target = 1ULL << (39 + epf);
        const u64 captured = sh_s(target);
        if (!inCheck || (captured & cm)) {
            u64 srcs = pawn_att_down(target) & c.pawns & c.mine;
            while (srcs) {
                const u64 s = srcs & (0 - srcs);
                srcs ^= s;
                if (s & pinned) {
                    if (!inCheck && (PG_TAB(line[ctz(s)][c.ksq]) & target)) n++;
                } else if (!ep_exposes_king(c, s, captured)) {
                    n++;
                }
            }
        }
    }

    // knights
    const u64 N = b.knights & c.mine & ~pinned;
    if (SvTraits<SV>::kogge && !PG_KNIGHT_LUT) {
        n += knight_set_count(N, targets);
    } else {
        u64 k = N;
        while (k) {
            n += popc(PG_TAB(knight[ctz(k)]) & targets);
            k &= k - 1;
        }
    }

    // sliders
    const u64 B = b.bq & c.mine & ~pinned;
    const u64 R = b.rq & c.mine & ~pinned;
    if (SvTraits<SV>::kogge) {
        constexpr int F = SvTraits<SV>::shift;
        n += ks_count_diag<F>(B, c.empty, targets) + ks_count_orth<F>(R, c.empty, targets);
    } else {
        u64 x = B;
        while (x) {
            n += popc(magic_bishop(ctz(x), c.occ) & targets);
            x &= x - 1;
        }
        x = R;
        while (x) {
            n += popc(magic_rook(ctz(x), c.occ) & targets);
            x &= x - 1;
        }
    }
    return n;
}

// ---------------------------------------------------------------- generate
// `from` may carry mover bits (bits 24-28) above the square.
PG_HD u32 encode_move(int from, int to, u32 flags)
{
    return (flags << 12) | ((u32)to << 6) | (u32)from;
}

// Emits every target square of a piece as a move.
template <class Sink>
PG_HD void emit_targets(Sink &out, int from, u64 targets)
{
    const u32 base = encode_move(from, 0, MF_QUIET);
    for_each_bit(targets, [&](int to) { out(base | ((u32)to << 6)); });
}

// Pawn move to dst with the four promotions on the last rank.
template <class Sink>
PG_HD void emit_pawn(Sink &out, int from, int to, u32 flags)
{
    if (to >= 56) {
        out(encode_move(from, to, MF_PROMO | 0));
        out(encode_move(from, to, MF_PROMO | 1));
        out(encode_move(from, to, MF_PROMO | 2));
        out(encode_move(from, to, MF_PROMO | 3));
    } else {
        out(encode_move(from, to, flags));
    }
}

// Mover bits (MOVER = true): each emitted move also carries, in bits 24-28,
// the planes the moving piece occupies (pawn 1, knight 2, bishop/queen 4,
// rook/queen 8, king 16), so make_child<true> needs no piece lookup.  The
// generator knows the piece of every move it emits, so the bits cost one OR
// per piece, not per move.
enum : u32 { MV_P = 1u << 24, MV_N = 2u << 24, MV_BQ = 4u << 24, MV_RQ = 8u << 24, MV_K = 16u << 24 };

// Generates every legal move of the side to move.  Emits exactly
// count_moves<SV>(b) moves.  GENSV >= 0 forces the slider variant of the
// per-piece targets and of the opponent's attack map.
template <int SV, bool MOVER = false, int GENSV = -1, class Sink>
PG_HD void gen_moves(const Board &b, Sink &out)
{
    // per-piece targets: one magic lookup per slider beats a single-bit
    // Kogge-Stone fill in every variant; the variant still decides the
    // set-wise opponent attack map
    constexpr int GEN_SV = GENSV >= 0 ? GENSV : (PG_GEN_MAGIC ? SV_MAGIC : SV);
    Ctx c;
    setup_ctx<GENSV >= 0 ? GENSV : (PG_GEN_MAGIC_ATTACKS ? GEN_SV : SV)>(b, c);
    const u64 notMine = ~c.mine;
    const u32 mvP = MOVER ? MV_P : 0, mvN = MOVER ? MV_N : 0, mvK = MOVER ? MV_K : 0;
    emit_targets(out, c.ksq | mvK, PG_TAB(king[c.ksq]) & notMine & ~c.attacked);
    const u64 cm = check_mask<SV>(c);
    if (!cm) return;
    const bool inCheck = cm != ~0ULL;
    const u64 targets = notMine & cm;

    if (!inCheck) {
        if ((c.st & 1) && !((c.occ | c.attacked) & 0x60ULL)) out(encode_move(4 | mvK, 6, MF_KING_CASTLE));
        if ((c.st & 2) && !(c.occ & 0x0EULL) && !(c.attacked & 0x0CULL)) out(encode_move(4 | mvK, 2, MF_QUEEN_CASTLE));
    }

    const u64 pinned = pinned_of(c);

    // pinned pieces: along the pin line only, never in check
    for_each_bit(inCheck ? 0 : pinned, [&](int s) {
        const u64 p = 1ULL << s;
        const u64 line = PG_TAB(line[s][c.ksq]);
        if (p & b.knights) return;
        if (p & c.pawns) {
            const u64 p1 = sh_n(p) & c.empty & line;
            if (p1) {
                out(encode_move(s | mvP, s + 8, MF_QUIET));
                if (sh_n(p1 & RANK3) & c.empty) out(encode_move(s | mvP, s + 16, MF_DOUBLE_PUSH));
            }
            const u64 cap = pawn_att_up(p) & line & c.theirs;
            if (cap) emit_pawn(out, s | mvP, ctz(cap), MF_CAPTURE);
            return;
        }
        u64 t = 0;
        if (p & b.bq) t |= bishop_att<GEN_SV>(s, c.occ);
        if (p & b.rq) t |= rook_att<GEN_SV>(s, c.occ);
        const u32 mv = MOVER ? (((p & b.bq) ? MV_BQ : 0u) | ((p & b.rq) ? MV_RQ : 0u)) : 0u;
        emit_targets(out, s | mv, t & notMine & line);
    });

    // free pieces
    for_each_bit(b.knights & c.mine & ~pinned,
                 [&](int s) { emit_targets(out, s | mvN, PG_TAB(knight[s]) & targets); });
    for_each_bit(b.bq & c.mine & ~pinned, [&](int s) {
        const u32 mv = MOVER ? (MV_BQ | (((b.rq >> s) & 1) ? MV_RQ : 0u)) : 0u;  // a queen is on both planes
        emit_targets(out, s | mv, bishop_att<GEN_SV>(s, c.occ) & targets);
    });
    for_each_bit(b.rq & c.mine & ~pinned, [&](int s) {
        const u32 mv = MOVER ? (MV_RQ | (((b.bq >> s) & 1) ? MV_BQ : 0u)) : 0u;
        emit_targets(out, s | mv, rook_att<GEN_SV>(s, c.occ) & targets);
    });
    const u64 P = c.pawns & c.mine & ~pinned;
    const u64 p1 = sh_n(P) & c.empty;
    u64 p1c = p1 & cm;
    u64 p2 = sh_n(p1 & RANK3) & c.empty & cm;
    for_each_bit(p1c, [&](int to) { emit_pawn(out, (to - 8) | mvP, to, MF_QUIET); });
    for_each_bit(p2, [&](int to) { out(encode_move((to - 16) | mvP, to, MF_DOUBLE_PUSH)); });
    const u64 capT = c.theirs & cm;
    for_each_bit(sh_nw(P) & capT, [&](int to) { emit_pawn(out, (to - 7) | mvP, to, MF_CAPTURE); });
    for_each_bit(sh_ne(P) & capT, [&](int to) { emit_pawn(out, (to - 9) | mvP, to, MF_CAPTURE); });
    const u32 epf = c.st >> 4;
    if (epf) {
        const u64 target = 1ULL << (39 + epf);
        const u64 captured = sh_s(target);
        if (!inCheck || (captured & cm)) {
            u64 srcs = pawn_att_down(target) & c.pawns & c.mine;
            while (srcs) {
                const u64 s = srcs & (0 - srcs);
                srcs ^= s;
                const bool ok = (s & pinned) ? (!inCheck && (PG_TAB(line[ctz(s)][c.ksq]) & target) != 0)
                                             : !ep_exposes_king(c, s, captured);
                if (ok) out(encode_move(ctz(s) | mvP, 39 + epf, MF_EP));
            }
        }
    }
}

// ------------------------------------------------------------------- make
// Applies a legal move and returns the child from the opponent's point of
// view (mirrored).  Branch-free except for the flag decode.
// With MOVER, mv carries the mover bits of gen_moves<SV, true> (bits 24-28)
// and the piece planes of the moving piece are not looked up; bits 16-23 are
// ignored either way.
template <bool MOVER = false>
PG_HD Board make_child(const Board &b, u32 mv)
{
    const int from = mv & 63, to = (mv >> 6) & 63;
    const u32 fl = (mv >> 12) & 15;
    const u64 src = PG_MAKE_TABLES ? PG_TAB(bit[from]) : 1ULL << from;
    const u64 dst = PG_MAKE_TABLES ? PG_TAB(bit[to]) : 1ULL << to;
    const u64 sd = src | dst;
    const u64 st = b.pawns & 0xFF;
    const u64 pawns0 = b.pawns & RANKS2TO7;
    const u64 theirPawns = pawns0 & ~b.mine;

    auto on = [&](u64 plane) -> u64 {  // all ones when the moving piece is on `plane`
        return PG_MAKE_TABLES ? maskIf((plane & src) != 0) : maskIf((plane >> from) & 1);
    };
    const u64 mP = MOVER ? maskIf(mv & MV_P) : on(pawns0);
    const u64 mN = MOVER ? maskIf(mv & MV_N) : on(b.knights);
    const u64 mB = MOVER ? maskIf(mv & MV_BQ) : on(b.bq);
    const u64 mR = MOVER ? maskIf(mv & MV_RQ) : on(b.rq);
    const u64 mK = MOVER ? maskIf(mv & MV_K) : on(b.kings);

    u64 pawns = pawns0 & ~sd;
    u64 kn = b.knights & ~sd;
    u64 bq = b.bq & ~sd;
    u64 rq = b.rq & ~sd;
    u64 kings = b.kings & ~src;

    const u64 mPromo = maskIf(fl & 8);
    const u32 pt = fl & 3;  // promotion piece: 0 N, 1 B, 2 R, 3 Q
    pawns |= dst & mP & ~mPromo;
    kn |= dst & ((mN & ~mPromo) | (mPromo & maskIf(pt == 0)));
    bq |= dst & ((mB & ~mPromo) | (mPromo & maskIf(pt == 1 || pt == 3)));
    rq |= dst & ((mR & ~mPromo) | (mPromo & maskIf(pt >= 2)));
    kings |= dst & mK;

    // en passant removes the pawn behind the target square
    pawns &= ~(sh_s(dst) & maskIf(fl == MF_EP));
    // castling moves the rook: h1->f1 or a1->d1
    const u64 rookHop = (fl == MF_KING_CASTLE) ? 0xA0ULL : (fl == MF_QUEEN_CASTLE ? 0x09ULL : 0ULL);
    rq ^= rookHop;
    const u64 mine = ((b.mine & ~src) | dst) ^ rookHop;

    // castling rights: king move, or anything leaving/landing on a rook corner
    u64 clear = PG_MAKE_TABLES
                    ? (mK & 3) | PG_TAB(castleClear[from]) | PG_TAB(castleClear[to])
                    : (mK & 3) | ((sd >> 7) & 1) | ((sd & 1) << 1) | ((sd >> 61) & 4) | ((sd >> 53) & 8);
    const u64 st2 = st & ~clear;

    // exact en-passant flagging: only when an enemy pawn stands beside dst
    u64 epf = 0;
    if (fl == MF_DOUBLE_PUSH && ((sh_e(dst) | sh_w(dst)) & theirPawns)) epf = (u64)((from & 7) + 1);

    const u64 occ = pawns | kn | bq | rq | kings;
    Board c;
    c.mine = flipv(occ & ~mine);
    c.pawns = flipv(pawns) | ((st2 >> 2) & 3) | ((st2 & 3) << 2) | (epf << 4) | ((~b.pawns) & SIDE_BIT);
    c.knights = flipv(kn);
    c.bq = flipv(bq);
    c.rq = flipv(rq);
    c.kings = flipv(kings);
    return c;
}

// The vertical mirror of every plane of a board (the parent in its child's
// frame).  The pawn plane's state byte moves to bits 56-63 and the side bit
// to bit 7, squares no pawn occupies.
PG_HD Board flip_board(const Board &b)
{
    return Board{flipv(b.mine), flipv(b.pawns), flipv(b.knights), flipv(b.bq), flipv(b.rq), flipv(b.kings)};
}

// make_child on the parent given mirrored (f = flip_board(parent)): the move
// is applied in the child's own frame, so the child needs no mirroring.
// Same result as make_child(flip_board(f), mv).  The move's squares are the
// parent's; in this frame they sit at square ^ 56, the parent's state byte
// at bits 56-63 and its side bit at bit 7.
PG_HD Board make_child_mirrored(const Board &f, u32 mv, int *moverKing = nullptr, int stillKing = 0,
                                u64 *occOut = nullptr, u64 *moverOut = nullptr)
{
    const int from = mv & 63, to = (mv >> 6) & 63;
    const u32 fl = (mv >> 12) & 15;
    const u64 src = PG_TAB(bit[from ^ 56]), dst = PG_TAB(bit[to ^ 56]);
    const u64 sd = src | dst;
    const u64 st = f.pawns >> 56;
    const u64 pawns0 = f.pawns & RANKS2TO7;
    const u64 theirPawns = pawns0 & ~f.mine;

    const u64 mP = maskIf((pawns0 & src) != 0);
    const u64 mN = maskIf((f.knights & src) != 0);
    const u64 mB = maskIf((f.bq & src) != 0);
    const u64 mR = maskIf((f.rq & src) != 0);
    const u64 mK = maskIf((f.kings & src) != 0);

    u64 pawns = pawns0 & ~sd;
    u64 kn = f.knights & ~sd;
    u64 bq = f.bq & ~sd;
    u64 rq = f.rq & ~sd;
    u64 kings = f.kings & ~src;

    const u64 mPromo = maskIf(fl & 8);
    const u32 pt = fl & 3;  // promotion piece: 0 N, 1 B, 2 R, 3 Q
    pawns |= dst & mP & ~mPromo;
    kn |= dst & ((mN & ~mPromo) | (mPromo & maskIf(pt == 0)));
    bq |= dst & ((mB & ~mPromo) | (mPromo & maskIf(pt == 1 || pt == 3)));
    rq |= dst & ((mR & ~mPromo) | (mPromo & maskIf(pt >= 2)));
    kings |= dst & mK;

    // en passant removes the pawn behind the target square (north of it here)
    pawns &= ~(sh_n(dst) & maskIf(fl == MF_EP));
    // castling moves the rook: h1->f1 or a1->d1 of the parent, on rank 8 here
    const u64 rookHop = (fl == MF_KING_CASTLE) ? (0xA0ULL << 56) : (fl == MF_QUEEN_CASTLE ? (0x09ULL << 56) : 0ULL);
    rq ^= rookHop;
    const u64 mine = ((f.mine & ~src) | dst) ^ rookHop;

    // castling rights: king move, or anything leaving/landing on a rook corner
    const u64 clear = (mK & 3) | PG_TAB(castleClear[from]) | PG_TAB(castleClear[to]);
    const u64 st2 = st & ~clear;

    // exact en-passant flagging: only when an enemy pawn stands beside dst
    u64 epf = 0;
    if (fl == MF_DOUBLE_PUSH && ((sh_e(dst) | sh_w(dst)) & theirPawns)) epf = (u64)((from & 7) + 1);

    // the moving side's king square in the child's frame, when asked: where a
    // king move lands, else `stillKing` (its square before the move)
    if (moverKing) *moverKing = mK ? (to ^ 56) : stillKing;

    const u64 occ = pawns | kn | bq | rq | kings;
    if (occOut) *occOut = occ;      // the child's occupancy
    if (moverOut) *moverOut = mine;  // the moving side's pieces: the child's opponent
    Board c;
    c.mine = occ & ~mine;
    c.pawns = pawns | ((st2 >> 2) & 3) | ((st2 & 3) << 2) | (epf << 4) | ((~f.pawns & 0x80ULL) << 56);
    c.knights = kn;
    c.bq = bq;
    c.rq = rq;
    c.kings = kings;
    return c;
}

// ---------------------------------------------------------- validation
// 0 when a pos48 board is a position the generator can search: piece planes
// disjoint (bishop and rook planes overlap only as queens), white pieces
// within the occupancy, one king per side, en-passant file 0..8, and the
// side not to move not in check.  The reference assumes all of this
// (a missing king makes its bit scans undefined), so it is checked here.
PG_HD int validate_pos48(const u64 p[6])
{
    const u64 pawns = p[1] & RANKS2TO7;
    const u64 sl = p[3] | p[4];
    const u64 occ = pawns | p[2] | sl | p[5];
    if ((pawns & p[2]) | (pawns & sl) | (pawns & p[5]) | (p[2] & sl) | (p[2] & p[5]) | (p[5] & sl)) return 1;
    if (p[0] & ~occ) return 2;
    if (popc(p[5] & p[0]) != 1 || popc(p[5] & ~p[0]) != 1) return 3;
    if (((p[1] >> 4) & 15) > 8) return 4;
    // the opponent's king must not be capturable
    const bool black = (p[1] >> 63) & 1;
    const u64 mine = black ? (occ & ~p[0]) : p[0];
    const u64 theirK = p[5] & ~mine;
    const u64 myP = pawns & mine;
    u64 att = (black ? pawn_att_down(myP) : pawn_att_up(myP)) | knight_set_att(p[2] & mine) |
              ks_diag(p[3] & mine, ~occ) | ks_orth(p[4] & mine, ~occ);
    const u64 k = p[5] & mine;
    att |= sh_n(k) | sh_s(k) | sh_e(k) | sh_w(k) | sh_ne(k) | sh_nw(k) | sh_se(k) | sh_sw(k);
    if (att & theirK) return 5;
    return 0;
}

// -------------------------------------------------- absolute <-> relative
// pos48: the reference's HexaBitBoardPosition (chess.h:208-230).
PG_HD Board from_pos48(const u64 p[6])
{
    const u64 state = p[1];
    const bool black = (state >> 63) & 1;
    const u64 pawns = state & RANKS2TO7;
    const u64 occ = pawns | p[2] | p[3] | p[4] | p[5];
    const u64 wc = state & 3, bc = (state >> 2) & 3, ep = (state >> 4) & 15;
    Board b;
    if (!black) {
        b.mine = p[0] & occ;
        b.pawns = pawns | wc | (bc << 2) | (ep << 4);
        b.knights = p[2];
        b.bq = p[3];
        b.rq = p[4];
        b.kings = p[5];
    } else {
        b.mine = flipv(occ & ~p[0]);
        b.pawns = flipv(pawns) | bc | (wc << 2) | (ep << 4) | SIDE_BIT;
        b.knights = flipv(p[2]);
        b.bq = flipv(p[3]);
        b.rq = flipv(p[4]);
        b.kings = flipv(p[5]);
    }
    return b;
}

PG_HD void to_pos48(const Board &b, u64 p[6])
{
    const bool black = (b.pawns >> 63) & 1;
    const u64 st = b.pawns & 0xFF;
    const u64 pawns = b.pawns & RANKS2TO7;
    const u64 occ = pawns | b.knights | b.bq | b.rq | b.kings;
    const u64 my = st & 3, their = (st >> 2) & 3, ep = (st >> 4) & 15;
    if (!black) {
        p[0] = b.mine;
        p[1] = pawns | my | (their << 2) | (ep << 4);
        p[2] = b.knights;
        p[3] = b.bq;
        p[4] = b.rq;
        p[5] = b.kings;
    } else {
        p[0] = flipv(occ & ~b.mine);
        p[1] = flipv(pawns) | their | (my << 2) | (ep << 4) | SIDE_BIT;
        p[2] = flipv(b.knights);
        p[3] = flipv(b.bq);
        p[4] = flipv(b.rq);
        p[5] = flipv(b.kings);
    }
}

}  // namespace pg
