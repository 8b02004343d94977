/* Test infrastructure: the perft ORACLE.
 *
 * A clean-room CPU restatement, in plain C, of the reference's host move
 * generator and perft (ankan-ban/perft_gpu).  It is the checker for the CUDA
 * engine: only tests/, the smoke check and bench.py's CPU-baseline leg may
 * load it.  The product never links or calls it.
 *
 * Parity pin: checked against the reference's own host perft compiled from
 * the reference sources (oracle/_ref/libperft_ref.so, built by
 * oracle/Makefile) and against the committed golden fixtures in tests/golden/
 * that were generated from that build.
 *
 * It follows the reference function by function:
 *   fills / attacks  MoveGeneratorBitboard.h:448-728 (Kogge-Stone sliders,
 *                    the reference's USE_SLIDING_LUT 0 variant)
 *   knight / king    MoveGeneratorBitboard.h:846-868
 *   between / line   MoveGeneratorBitboard.h:895-963 (tables, init :1021-1031)
 *   pins             findPinnedPieces     MoveGeneratorBitboard.h:1213-1249
 *   attacked map     findAttackedSquares  MoveGeneratorBitboard.h:1254-1298
 *   count            countMoves           MoveGeneratorBitboard.h:3008-3295
 *                    countMovesOutOfCheck MoveGeneratorBitboard.h:2828-3002
 *   generate         generateMoves        MoveGeneratorBitboard.h:2471-2823
 *                    generateMovesOutOfCheck MoveGeneratorBitboard.h:2269-2465
 *                    addCompactPawnMoves  MoveGeneratorBitboard.h:1723-1738
 *   make             makeMove (no hash)   MoveGeneratorBitboard.h:3310-3570
 *                    updateCastleFlag     MoveGeneratorBitboard.h:1310-1340
 *                    (EXACT_EN_PASSENT_FLAGGING, switches.h:48)
 *   perft            leaf count at depth 1 as in perft_bb.h:79-101 and the
 *                    GPU BFS (perft_bb.h:1027-1138)
 *   FEN              Utils::readFENString util.cpp:189-281 (clocks ignored),
 *                    Utils::board088ToHexBB util.cpp:92-140
 *
 * Compiled as C++ with -DORACLE_OPCOUNT, the same source counts the 64-bit
 * integer operations it executes (see opcount_main.cpp).  In that build each
 * slider lookup is charged at the reference's default fancy-magic cost
 * (MoveGeneratorBitboard.h:731-747: bit scan, not, and, multiply, shift, add)
 * instead of the Kogge-Stone fill used here for the value.
 */
#include "perft_oracle.h"

#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_OPCOUNT
#include "opcount.hpp"
#else
#include <pthread.h>
typedef uint64_t U64;
#define OPS(n) ((void)0)
static inline int popc(U64 x) { return __builtin_popcountll(x); }
static inline int ctz(U64 x) { return __builtin_ctzll(x); }
static inline uint64_t RAW(U64 x) { return x; }
#endif

#define WHITE 0
#define BLACK 1

#define RANKS2TO7 0x00FFFFFFFFFFFF00ULL
#define RANK1 0x00000000000000FFULL
#define RANK3 0x0000000000FF0000ULL
#define RANK8 0xFF00000000000000ULL
#define FILEA 0x0101010101010101ULL
#define FILEH 0x8080808080808080ULL
#define F1G1 0x60ULL
#define C1D1 0x0CULL
#define B1D1 0x0EULL
#define F8G8 0x6000000000000000ULL
#define C8D8 0x0C00000000000000ULL
#define B8D8 0x0E00000000000000ULL

/* CMove flag codes (chess.h:269-293) */
#define FL_QUIET 0
#define FL_DOUBLE_PUSH 1
#define FL_KING_CASTLE 2
#define FL_QUEEN_CASTLE 3
#define FL_CAPTURE 4
#define FL_EP_CAPTURE 5
#define FL_PROMO_N 8
#define FL_PROMO_B 9
#define FL_PROMO_R 10
#define FL_PROMO_Q 11

enum { P_WHITE = 0, P_PAWNS, P_KNIGHTS, P_BQ, P_RQ, P_KINGS };

/* ---------------------------------------------------------------- state */

static inline int st_chance(const oracle_pos *p) { return (int)(p->bb[P_PAWNS] >> 63); }
static inline int st_wcastle(const oracle_pos *p) { return (int)(p->bb[P_PAWNS] & 3); }
static inline int st_bcastle(const oracle_pos *p) { return (int)((p->bb[P_PAWNS] >> 2) & 3); }
static inline int st_ep(const oracle_pos *p) { return (int)((p->bb[P_PAWNS] >> 4) & 15); }

static inline void st_set_chance(oracle_pos *p, int c)
{
    p->bb[P_PAWNS] = (p->bb[P_PAWNS] & ~(1ULL << 63)) | ((uint64_t)(c & 1) << 63);
}
static inline void st_set_wcastle(oracle_pos *p, int v)
{
    p->bb[P_PAWNS] = (p->bb[P_PAWNS] & ~3ULL) | (uint64_t)(v & 3);
}
static inline void st_set_bcastle(oracle_pos *p, int v)
{
    p->bb[P_PAWNS] = (p->bb[P_PAWNS] & ~(3ULL << 2)) | ((uint64_t)(v & 3) << 2);
}
static inline void st_set_ep(oracle_pos *p, int v)
{
    p->bb[P_PAWNS] = (p->bb[P_PAWNS] & ~(15ULL << 4)) | ((uint64_t)(v & 15) << 4);
}

/* ------------------------------------------------------- one-step shifts */
/* MoveGeneratorBitboard.h:448-486 */
static inline U64 northOne(U64 x) { return x << 8; }
static inline U64 southOne(U64 x) { return x >> 8; }
static inline U64 eastOne(U64 x) { return (x << 1) & ~FILEA; }
static inline U64 westOne(U64 x) { return (x >> 1) & ~FILEH; }
static inline U64 northEastOne(U64 x) { return (x << 9) & ~FILEA; }
static inline U64 northWestOne(U64 x) { return (x << 7) & ~FILEH; }
static inline U64 southEastOne(U64 x) { return (x >> 7) & ~FILEA; }
static inline U64 southWestOne(U64 x) { return (x >> 9) & ~FILEH; }

/* ------------------------------------------------ Kogge-Stone fills (raw) */
/* MoveGeneratorBitboard.h:504-700.  Occluded fill of gen through pro, then
 * one more step: the attack set in that direction.  These run on raw
 * integers; the op-counting build charges them at the magic-lookup cost. */
typedef uint64_t R64;
static inline R64 ks_n(R64 g, R64 p)
{
    g |= (g << 8) & p; p &= p << 8; g |= (g << 16) & p; p &= p << 16; g |= (g << 32) & p;
    return g << 8;
}
static inline R64 ks_s(R64 g, R64 p)
{
    g |= (g >> 8) & p; p &= p >> 8; g |= (g >> 16) & p; p &= p >> 16; g |= (g >> 32) & p;
    return g >> 8;
}
static inline R64 ks_e(R64 g, R64 p)
{
    p &= ~FILEA;
    g |= (g << 1) & p; p &= p << 1; g |= (g << 2) & p; p &= p << 2; g |= (g << 4) & p;
    return (g << 1) & ~FILEA;
}
static inline R64 ks_w(R64 g, R64 p)
{
    p &= ~FILEH;
    g |= (g >> 1) & p; p &= p >> 1; g |= (g >> 2) & p; p &= p >> 2; g |= (g >> 4) & p;
    return (g >> 1) & ~FILEH;
}
static inline R64 ks_ne(R64 g, R64 p)
{
    p &= ~FILEA;
    g |= (g << 9) & p; p &= p << 9; g |= (g << 18) & p; p &= p << 18; g |= (g << 36) & p;
    return (g << 9) & ~FILEA;
}
static inline R64 ks_nw(R64 g, R64 p)
{
    p &= ~FILEH;
    g |= (g << 7) & p; p &= p << 7; g |= (g << 14) & p; p &= p << 14; g |= (g << 28) & p;
    return (g << 7) & ~FILEH;
}
static inline R64 ks_se(R64 g, R64 p)
{
    p &= ~FILEA;
    g |= (g >> 7) & p; p &= p >> 7; g |= (g >> 14) & p; p &= p >> 14; g |= (g >> 28) & p;
    return (g >> 7) & ~FILEA;
}
static inline R64 ks_sw(R64 g, R64 p)
{
    p &= ~FILEH;
    g |= (g >> 9) & p; p &= p >> 9; g |= (g >> 18) & p; p &= p >> 18; g |= (g >> 36) & p;
    return (g >> 9) & ~FILEH;
}

/* Attacks of ONE slider (MoveGeneratorBitboard.h:731-829 semantics). */
static inline U64 bishopAttacks(U64 piece, U64 pro)
{
    R64 g = RAW(piece), p = RAW(pro);
    OPS(6);
    return (U64)(ks_ne(g, p) | ks_nw(g, p) | ks_se(g, p) | ks_sw(g, p));
}
static inline U64 rookAttacks(U64 piece, U64 pro)
{
    R64 g = RAW(piece), p = RAW(pro);
    OPS(6);
    return (U64)(ks_n(g, p) | ks_s(g, p) | ks_e(g, p) | ks_w(g, p));
}
/* East+west rays of a set (used raw for the ep horizontal-pin test,
 * MoveGeneratorBitboard.h:3079-3082: the reference uses the Kogge-Stone
 * fills there in every build, so they are counted as such). */
static inline U64 eastWestAttacks(U64 rooks, U64 pro)
{
    R64 g = RAW(rooks), p = RAW(pro);
    OPS(2 * 13 + 1);
    return (U64)(ks_e(g, p) | ks_w(g, p));
}

static inline U64 getOne(U64 x) { return x & (0 - x); }
static inline int isSingular(U64 x) { return !(x ^ getOne(x)); }

/* multiBishopAttacks / multiRookAttacks: one lookup per piece
 * (MoveGeneratorBitboard.h:796-828). */
static inline U64 multiBishopAttacks(U64 bishops, U64 pro)
{
    U64 a = 0;
    while (bishops) {
        U64 b = getOne(bishops);
        a |= bishopAttacks(b, pro);
        bishops ^= b;
    }
    return a;
}
static inline U64 multiRookAttacks(U64 rooks, U64 pro)
{
    U64 a = 0;
    while (rooks) {
        U64 r = getOne(rooks);
        a |= rookAttacks(r, pro);
        rooks ^= r;
    }
    return a;
}

/* MoveGeneratorBitboard.h:846-868 */
static inline U64 kingAttacksSet(U64 k)
{
    U64 a = eastOne(k) | westOne(k);
    k |= a;
    a |= northOne(k) | southOne(k);
    return a;
}
static inline U64 knightAttacksSet(U64 n)
{
    U64 l1 = (n >> 1) & 0x7f7f7f7f7f7f7f7fULL;
    U64 l2 = (n >> 2) & 0x3f3f3f3f3f3f3f3fULL;
    U64 r1 = (n << 1) & 0xfefefefefefefefeULL;
    U64 r2 = (n << 2) & 0xfcfcfcfcfcfcfcfcULL;
    U64 h1 = l1 | r1;
    U64 h2 = l2 | r2;
    return (h1 << 16) | (h1 >> 16) | (h2 << 8) | (h2 >> 8);
}

/* ----------------------------------------------------------------- tables */
static uint64_t T_BETWEEN[64][64];
static uint64_t T_LINE[64][64];
static uint64_t T_ROOK[64], T_BISHOP[64], T_KING[64], T_KNIGHT[64];
static int g_ready;

/* Squares strictly between a and b on a common rank/file/diagonal, else 0. */
static uint64_t between_calc(int a, int b)
{
    int fa = a & 7, ra = a >> 3, fb = b & 7, rb = b >> 3;
    int df = (fb > fa) - (fb < fa), dr = (rb > ra) - (rb < ra);
    if (a == b) return 0;
    if (!(fa == fb || ra == rb || (fb - fa) == (rb - ra) || (fb - fa) == -(rb - ra))) return 0;
    uint64_t m = 0;
    int f = fa + df, r = ra + dr;
    while (f != fb || r != rb) {
        m |= 1ULL << (r * 8 + f);
        f += df;
        r += dr;
    }
    return m;
}

/* The whole rank/file/diagonal through a and b (both included), else 0. */
static uint64_t line_calc(int a, int b)
{
    int fa = a & 7, ra = a >> 3, fb = b & 7, rb = b >> 3;
    int df, dr;
    if (a == b) return 0;
    if (fa == fb) { df = 0; dr = 1; }
    else if (ra == rb) { df = 1; dr = 0; }
    else if ((fb - fa) == (rb - ra)) { df = 1; dr = 1; }
    else if ((fb - fa) == -(rb - ra)) { df = 1; dr = -1; }
    else return 0;
    uint64_t m = 1ULL << a;
    for (int s = -1; s <= 1; s += 2) {
        int f = fa + s * df, r = ra + s * dr;
        while (f >= 0 && f < 8 && r >= 0 && r < 8) {
            m |= 1ULL << (r * 8 + f);
            f += s * df;
            r += s * dr;
        }
    }
    return m;
}

int oracle_init(void)
{
    if (g_ready) return 0;
    for (int s = 0; s < 64; s++) {
        R64 x = 1ULL << s, all = ~0ULL;
        T_ROOK[s] = ks_n(x, all) | ks_s(x, all) | ks_e(x, all) | ks_w(x, all);
        T_BISHOP[s] = ks_ne(x, all) | ks_nw(x, all) | ks_se(x, all) | ks_sw(x, all);
        T_KING[s] = RAW(kingAttacksSet((U64)x));
        T_KNIGHT[s] = RAW(knightAttacksSet((U64)x));
        for (int t = 0; t < 64; t++) {
            T_BETWEEN[s][t] = between_calc(s, t);
            T_LINE[s][t] = line_calc(s, t);
        }
    }
    g_ready = 1;
    return 0;
}

/* ------------------------------------------------------- pins and threats */

/* findPinnedPieces, MoveGeneratorBitboard.h:1213-1249 */
static U64 findPinnedPieces(U64 enemyBishops, U64 enemyRooks, U64 allPieces, int kingIndex)
{
    U64 attackers = ((U64)T_BISHOP[kingIndex] & enemyBishops) | ((U64)T_ROOK[kingIndex] & enemyRooks);
    U64 pinned = 0;
    while (attackers) {
        U64 attacker = getOne(attackers);
        int ai = ctz(attacker);
        U64 inBetween = (U64)T_BETWEEN[ai][kingIndex] & allPieces;
        if (isSingular(inBetween)) pinned |= inBetween;
        attackers ^= attacker;
    }
    return pinned;
}

/* findAttackedSquares, MoveGeneratorBitboard.h:1254-1298.  The own king is
 * transparent to enemy sliders. */
static U64 findAttackedSquares(U64 emptySquares, U64 enemyBishops, U64 enemyRooks, U64 enemyPawns,
                               U64 enemyKnights, U64 enemyKing, U64 myKing, int enemyColor)
{
    U64 attacked = 0;
    if (enemyColor == WHITE)
        attacked |= northEastOne(enemyPawns) | northWestOne(enemyPawns);
    else
        attacked |= southEastOne(enemyPawns) | southWestOne(enemyPawns);
    attacked |= knightAttacksSet(enemyKnights);
    attacked |= multiBishopAttacks(enemyBishops, emptySquares | myKing);
    attacked |= multiRookAttacks(enemyRooks, emptySquares | myKing);
    attacked |= kingAttacksSet(enemyKing);
    return attacked;
}

typedef struct {
    U64 allPawns, allPieces, myPieces, enemyPieces, enemyBishops, enemyRooks;
    U64 myKing, pinned, threatened;
    int kingIndex, chance;
} ctx_t;

static void setup(const oracle_pos *pos, ctx_t *c)
{
    int chance = st_chance(pos);
    U64 allPawns = (U64)pos->bb[P_PAWNS] & RANKS2TO7;
    U64 allPieces = (U64)pos->bb[P_KINGS] | allPawns | (U64)pos->bb[P_KNIGHTS] |
                    (U64)pos->bb[P_BQ] | (U64)pos->bb[P_RQ];
    U64 blackPieces = allPieces & ~(U64)pos->bb[P_WHITE];
    U64 myPieces = chance == WHITE ? (U64)pos->bb[P_WHITE] : blackPieces;
    U64 enemyPieces = chance == WHITE ? blackPieces : (U64)pos->bb[P_WHITE];
    c->chance = chance;
    c->allPawns = allPawns;
    c->allPieces = allPieces;
    c->myPieces = myPieces;
    c->enemyPieces = enemyPieces;
    c->enemyBishops = (U64)pos->bb[P_BQ] & enemyPieces;
    c->enemyRooks = (U64)pos->bb[P_RQ] & enemyPieces;
    c->myKing = (U64)pos->bb[P_KINGS] & myPieces;
    c->kingIndex = ctz(c->myKing);
    c->pinned = findPinnedPieces(c->enemyBishops, c->enemyRooks, allPieces, c->kingIndex);
    c->threatened = findAttackedSquares(~allPieces, c->enemyBishops, c->enemyRooks,
                                        allPawns & enemyPieces, (U64)pos->bb[P_KNIGHTS] & enemyPieces,
                                        (U64)pos->bb[P_KINGS] & enemyPieces, c->myKing, !chance);
}

static U64 epTargetOf(const oracle_pos *pos, int chance)
{
    int ep = st_ep(pos);
    if (!ep) return 0;
    return chance == BLACK ? (1ULL << (ep - 1)) << 16 : (1ULL << (ep - 1)) << 40;
}

/* Single checker set (pawn, knight, slider) of the side to move's king,
 * MoveGeneratorBitboard.h:2838-2858. */
static U64 checkersOf(const oracle_pos *pos, const ctx_t *c)
{
    U64 king = c->myKing, attackers = 0;
    U64 enemyPawns = c->allPawns & c->enemyPieces;
    attackers |= (c->chance == WHITE ? (northEastOne(king) | northWestOne(king))
                                     : (southEastOne(king) | southWestOne(king))) & enemyPawns;
    attackers |= knightAttacksSet(king) & ((U64)pos->bb[P_KNIGHTS] & c->enemyPieces);
    attackers |= bishopAttacks(king, ~c->allPieces) & c->enemyBishops;
    attackers |= rookAttacks(king, ~c->allPieces) & c->enemyRooks;
    return attackers;
}

/* ------------------------------------------------------------------ count */

/* countMovesOutOfCheck, MoveGeneratorBitboard.h:2828-3002 */
static uint32_t countOutOfCheck(const oracle_pos *pos, const ctx_t *c)
{
    uint32_t n = 0;
    int chance = c->chance;
    U64 attackers = checkersOf(pos, c);
    U64 kingMoves = (U64)T_KING[c->kingIndex] & ~(c->threatened | c->myPieces);
    n += popc(kingMoves);
    if (!isSingular(attackers)) return n;

    U64 safe = attackers | (U64)T_BETWEEN[c->kingIndex][ctz(attackers)];
    U64 myPieces = c->myPieces & ~c->pinned;
    U64 myPawns = c->allPawns & myPieces;
    U64 dblRank = (U64)RANK3 << (chance * 24);
    U64 epTarget = epTargetOf(pos, chance);
    U64 epCaptured = chance == WHITE ? southOne(epTarget) : northOne(epTarget);
    if (epCaptured != attackers) epTarget = 0;

    while (myPawns) {
        U64 pawn = getOne(myPawns);
        U64 dst = (chance == WHITE ? northOne(pawn) : southOne(pawn)) & ~c->allPieces;
        if (dst) {
            if (dst & safe) {
                n += (dst & (RANK1 | RANK8)) ? 4 : 1;
            } else {
                dst = (chance == WHITE ? northOne(dst & dblRank) : southOne(dst & dblRank)) & safe & ~c->allPieces;
                if (dst) n++;
            }
        }
        U64 w = chance == WHITE ? northWestOne(pawn) : southWestOne(pawn);
        U64 e = chance == WHITE ? northEastOne(pawn) : southEastOne(pawn);
        dst = (w | e) & c->enemyPieces & safe;
        if (dst) n += (dst & (RANK1 | RANK8)) ? 4 : 1;
        dst = (w | e) & epTarget;
        if (dst) n++;
        myPawns ^= pawn;
    }
    U64 knights = (U64)pos->bb[P_KNIGHTS] & myPieces;
    while (knights) {
        U64 k = getOne(knights);
        n += popc((U64)T_KNIGHT[ctz(k)] & safe);
        knights ^= k;
    }
    U64 bishops = (U64)pos->bb[P_BQ] & myPieces;
    while (bishops) {
        U64 b = getOne(bishops);
        n += popc(bishopAttacks(b, ~c->allPieces) & safe);
        bishops ^= b;
    }
    U64 rooks = (U64)pos->bb[P_RQ] & myPieces;
    while (rooks) {
        U64 r = getOne(rooks);
        n += popc(rookAttacks(r, ~c->allPieces) & safe);
        rooks ^= r;
    }
    return n;
}

/* countMoves, MoveGeneratorBitboard.h:3008-3295 */
static uint32_t countMovesImpl(const oracle_pos *pos)
{
    ctx_t c;
    setup(pos, &c);
    if (c.threatened & c.myKing) return countOutOfCheck(pos, &c);

    int chance = c.chance;
    uint32_t n = 0;
    U64 myPawns = c.allPawns & c.myPieces;

    /* en passant (MoveGeneratorBitboard.h:3054-3092) */
    U64 epTarget = epTargetOf(pos, chance);
    if (epTarget) {
        U64 epCaptured = chance == WHITE ? southOne(epTarget) : northOne(epTarget);
        U64 epSources = (eastOne(epCaptured) | westOne(epCaptured)) & myPawns;
        while (epSources) {
            U64 pawn = getOne(epSources);
            if (pawn & c.pinned) {
                if (epTarget & (U64)T_LINE[ctz(pawn)][c.kingIndex]) n++;
            } else {
                U64 pro = ~c.allPieces | epCaptured | pawn;
                if (!(eastWestAttacks(c.enemyRooks, pro) & c.myKing)) n++;
            }
            epSources ^= pawn;
        }
    }

    U64 dblRank = (U64)RANK3 << (chance * 24);

    /* pinned pawns (MoveGeneratorBitboard.h:3099-3136) */
    U64 pinnedPawns = myPawns & c.pinned;
    while (pinnedPawns) {
        U64 pawn = getOne(pinnedPawns);
        U64 line = (U64)T_LINE[ctz(pawn)][c.kingIndex];
        U64 dst = (chance == WHITE ? northOne(pawn) : southOne(pawn)) & line & ~c.allPieces;
        if (dst) {
            n++;
            dst = (chance == WHITE ? northOne(dst & dblRank) : southOne(dst & dblRank)) & ~c.allPieces;
            if (dst) n++;
        }
        dst = (chance == WHITE ? northWestOne(pawn) : southWestOne(pawn)) & line;
        dst |= (chance == WHITE ? northEastOne(pawn) : southEastOne(pawn)) & line;
        if (dst & c.enemyPieces) n += (dst & (RANK1 | RANK8)) ? 4 : 1;
        pinnedPawns ^= pawn;
    }

    /* free pawns, set-wise (MoveGeneratorBitboard.h:3138-3166) */
    myPawns &= ~c.pinned;
    U64 dsts = (chance == WHITE ? northOne(myPawns) : southOne(myPawns)) & ~c.allPieces;
    n += popc(dsts);
    n += 3 * popc(dsts & (RANK1 | RANK8));
    dsts = (chance == WHITE ? northOne(dsts & dblRank) : southOne(dsts & dblRank)) & ~c.allPieces;
    n += popc(dsts);
    dsts = (chance == WHITE ? northWestOne(myPawns) : southWestOne(myPawns)) & c.enemyPieces;
    n += popc(dsts);
    n += 3 * popc(dsts & (RANK1 | RANK8));
    dsts = (chance == WHITE ? northEastOne(myPawns) : southEastOne(myPawns)) & c.enemyPieces;
    n += popc(dsts);
    n += 3 * popc(dsts & (RANK1 | RANK8));

    /* castling (MoveGeneratorBitboard.h:3168-3208) */
    if (chance == WHITE) {
        int wc = st_wcastle(pos);
        if ((wc & 1) && !(F1G1 & c.allPieces) && !(F1G1 & c.threatened)) n++;
        if ((wc & 2) && !(B1D1 & c.allPieces) && !(C1D1 & c.threatened)) n++;
    } else {
        int bc = st_bcastle(pos);
        if ((bc & 1) && !(F8G8 & c.allPieces) && !(F8G8 & c.threatened)) n++;
        if ((bc & 2) && !(B8D8 & c.allPieces) && !(C8D8 & c.threatened)) n++;
    }

    /* king (MoveGeneratorBitboard.h:3210-3218) */
    n += popc((U64)T_KING[c.kingIndex] & ~(c.threatened | c.myPieces));

    /* knights, not pinned (MoveGeneratorBitboard.h:3220-3233) */
    U64 knights = (U64)pos->bb[P_KNIGHTS] & c.myPieces & ~c.pinned;
    while (knights) {
        U64 k = getOne(knights);
        n += popc((U64)T_KNIGHT[ctz(k)] & ~c.myPieces);
        knights ^= k;
    }

    /* bishops/queens then rooks/queens, pinned ones restricted to the king
     * line (MoveGeneratorBitboard.h:3236-3292) */
    U64 myB = (U64)pos->bb[P_BQ] & c.myPieces;
    U64 b = myB & c.pinned;
    while (b) {
        U64 x = getOne(b);
        n += popc(bishopAttacks(x, ~c.allPieces) & ~c.myPieces & (U64)T_LINE[ctz(x)][c.kingIndex]);
        b ^= x;
    }
    b = myB & ~c.pinned;
    while (b) {
        U64 x = getOne(b);
        n += popc(bishopAttacks(x, ~c.allPieces) & ~c.myPieces);
        b ^= x;
    }
    U64 myR = (U64)pos->bb[P_RQ] & c.myPieces;
    U64 r = myR & c.pinned;
    while (r) {
        U64 x = getOne(r);
        n += popc(rookAttacks(x, ~c.allPieces) & ~c.myPieces & (U64)T_LINE[ctz(x)][c.kingIndex]);
        r ^= x;
    }
    r = myR & ~c.pinned;
    while (r) {
        U64 x = getOne(r);
        n += popc(rookAttacks(x, ~c.allPieces) & ~c.myPieces);
        r ^= x;
    }
    return n;
}

uint32_t oracle_count_moves(const oracle_pos *pos)
{
    if (!g_ready) oracle_init();
    return countMovesImpl(pos);
}

/* --------------------------------------------------------------- generate */

typedef struct {
    uint16_t *out;
    uint32_t n;
} mlist;

static inline void addMove(mlist *l, int from, int to, int flags)
{
    l->out[l->n++] = (uint16_t)(((flags & 15) << 12) | ((to & 63) << 6) | (from & 63));
}

/* addCompactPawnMoves, MoveGeneratorBitboard.h:1723-1738 */
static inline void addPawnMoves(mlist *l, int from, U64 dst, int flags)
{
    int to = ctz(dst);
    if (dst & (RANK1 | RANK8)) {
        addMove(l, from, to, flags | FL_PROMO_N);
        addMove(l, from, to, flags | FL_PROMO_B);
        addMove(l, from, to, flags | FL_PROMO_Q);
        addMove(l, from, to, flags | FL_PROMO_R);
    } else {
        addMove(l, from, to, flags);
    }
}

static void addTargets(mlist *l, int from, U64 targets)
{
    while (targets) {
        U64 d = getOne(targets);
        addMove(l, from, ctz(d), FL_QUIET);
        targets ^= d;
    }
}

/* generateMovesOutOfCheck, MoveGeneratorBitboard.h:2269-2465 */
static void genOutOfCheck(const oracle_pos *pos, const ctx_t *c, mlist *l)
{
    int chance = c->chance;
    U64 attackers = checkersOf(pos, c);
    addTargets(l, c->kingIndex, (U64)T_KING[c->kingIndex] & ~(c->threatened | c->myPieces));
    if (!isSingular(attackers)) return;

    U64 safe = attackers | (U64)T_BETWEEN[c->kingIndex][ctz(attackers)];
    U64 myPieces = c->myPieces & ~c->pinned;
    U64 myPawns = c->allPawns & myPieces;
    U64 dblRank = (U64)RANK3 << (chance * 24);
    U64 epTarget = epTargetOf(pos, chance);
    U64 epCaptured = chance == WHITE ? southOne(epTarget) : northOne(epTarget);
    if (epCaptured != attackers) epTarget = 0;

    while (myPawns) {
        U64 pawn = getOne(myPawns);
        int from = ctz(pawn);
        U64 dst = (chance == WHITE ? northOne(pawn) : southOne(pawn)) & ~c->allPieces;
        if (dst) {
            if (dst & safe) {
                addPawnMoves(l, from, dst, 0);
            } else {
                dst = (chance == WHITE ? northOne(dst & dblRank) : southOne(dst & dblRank)) & safe & ~c->allPieces;
                if (dst) addMove(l, from, ctz(dst), FL_DOUBLE_PUSH);
            }
        }
        U64 w = chance == WHITE ? northWestOne(pawn) : southWestOne(pawn);
        U64 e = chance == WHITE ? northEastOne(pawn) : southEastOne(pawn);
        dst = (w | e) & c->enemyPieces & safe;
        if (dst) addPawnMoves(l, from, dst, FL_CAPTURE);
        dst = (w | e) & epTarget;
        if (dst) addMove(l, from, ctz(dst), FL_EP_CAPTURE);
        myPawns ^= pawn;
    }
    U64 knights = (U64)pos->bb[P_KNIGHTS] & myPieces;
    while (knights) {
        U64 k = getOne(knights);
        addTargets(l, ctz(k), (U64)T_KNIGHT[ctz(k)] & safe);
        knights ^= k;
    }
    U64 bishops = (U64)pos->bb[P_BQ] & myPieces;
    while (bishops) {
        U64 b = getOne(bishops);
        addTargets(l, ctz(b), bishopAttacks(b, ~c->allPieces) & safe);
        bishops ^= b;
    }
    U64 rooks = (U64)pos->bb[P_RQ] & myPieces;
    while (rooks) {
        U64 r = getOne(rooks);
        addTargets(l, ctz(r), rookAttacks(r, ~c->allPieces) & safe);
        rooks ^= r;
    }
}

/* generateMoves, MoveGeneratorBitboard.h:2471-2823 */
uint32_t oracle_generate_moves(const oracle_pos *pos, uint16_t *moves)
{
    ctx_t c;
    mlist l;
    if (!g_ready) oracle_init();
    l.out = moves;
    l.n = 0;
    setup(pos, &c);
    if (c.threatened & c.myKing) {
        genOutOfCheck(pos, &c, &l);
        return l.n;
    }
    int chance = c.chance;

    addTargets(&l, c.kingIndex, (U64)T_KING[c.kingIndex] & ~(c.threatened | c.myPieces));

    U64 knights = (U64)pos->bb[P_KNIGHTS] & c.myPieces & ~c.pinned;
    while (knights) {
        U64 k = getOne(knights);
        addTargets(&l, ctz(k), (U64)T_KNIGHT[ctz(k)] & ~c.myPieces);
        knights ^= k;
    }

    U64 myB = (U64)pos->bb[P_BQ] & c.myPieces;
    U64 b = myB & c.pinned;
    while (b) {
        U64 x = getOne(b);
        addTargets(&l, ctz(x), bishopAttacks(x, ~c.allPieces) & ~c.myPieces & (U64)T_LINE[ctz(x)][c.kingIndex]);
        b ^= x;
    }
    b = myB & ~c.pinned;
    while (b) {
        U64 x = getOne(b);
        addTargets(&l, ctz(x), bishopAttacks(x, ~c.allPieces) & ~c.myPieces);
        b ^= x;
    }
    U64 myR = (U64)pos->bb[P_RQ] & c.myPieces;
    U64 r = myR & c.pinned;
    while (r) {
        U64 x = getOne(r);
        addTargets(&l, ctz(x), rookAttacks(x, ~c.allPieces) & ~c.myPieces & (U64)T_LINE[ctz(x)][c.kingIndex]);
        r ^= x;
    }
    r = myR & ~c.pinned;
    while (r) {
        U64 x = getOne(r);
        addTargets(&l, ctz(x), rookAttacks(x, ~c.allPieces) & ~c.myPieces);
        r ^= x;
    }

    U64 myPawns = c.allPawns & c.myPieces;

    U64 epTarget = epTargetOf(pos, chance);
    if (epTarget) {
        U64 epCaptured = chance == WHITE ? southOne(epTarget) : northOne(epTarget);
        U64 epSources = (eastOne(epCaptured) | westOne(epCaptured)) & myPawns;
        while (epSources) {
            U64 pawn = getOne(epSources);
            if (pawn & c.pinned) {
                if (epTarget & (U64)T_LINE[ctz(pawn)][c.kingIndex])
                    addMove(&l, ctz(pawn), ctz(epTarget), FL_EP_CAPTURE);
            } else {
                U64 pro = ~c.allPieces | epCaptured | pawn;
                if (!(eastWestAttacks(c.enemyRooks, pro) & c.myKing))
                    addMove(&l, ctz(pawn), ctz(epTarget), FL_EP_CAPTURE);
            }
            epSources ^= pawn;
        }
    }

    U64 dblRank = (U64)RANK3 << (chance * 24);
    U64 pinnedPawns = myPawns & c.pinned;
    while (pinnedPawns) {
        U64 pawn = getOne(pinnedPawns);
        int from = ctz(pawn);
        U64 line = (U64)T_LINE[from][c.kingIndex];
        U64 dst = (chance == WHITE ? northOne(pawn) : southOne(pawn)) & line & ~c.allPieces;
        if (dst) {
            addMove(&l, from, ctz(dst), FL_QUIET);
            dst = (chance == WHITE ? northOne(dst & dblRank) : southOne(dst & dblRank)) & ~c.allPieces;
            if (dst) addMove(&l, from, ctz(dst), FL_DOUBLE_PUSH);
        }
        dst = (chance == WHITE ? northWestOne(pawn) : southWestOne(pawn)) & line;
        dst |= (chance == WHITE ? northEastOne(pawn) : southEastOne(pawn)) & line;
        if (dst & c.enemyPieces) addPawnMoves(&l, from, dst, FL_CAPTURE);
        pinnedPawns ^= pawn;
    }
    myPawns &= ~c.pinned;
    while (myPawns) {
        U64 pawn = getOne(myPawns);
        int from = ctz(pawn);
        U64 dst = (chance == WHITE ? northOne(pawn) : southOne(pawn)) & ~c.allPieces;
        if (dst) {
            addPawnMoves(&l, from, dst, 0);
            dst = (chance == WHITE ? northOne(dst & dblRank) : southOne(dst & dblRank)) & ~c.allPieces;
            if (dst) addPawnMoves(&l, from, dst, FL_DOUBLE_PUSH);
        }
        U64 w = (chance == WHITE ? northWestOne(pawn) : southWestOne(pawn)) & c.enemyPieces;
        if (w) addPawnMoves(&l, from, w, FL_CAPTURE);
        U64 e = (chance == WHITE ? northEastOne(pawn) : southEastOne(pawn)) & c.enemyPieces;
        if (e) addPawnMoves(&l, from, e, FL_CAPTURE);
        myPawns ^= pawn;
    }

    if (chance == WHITE) {
        int wc = st_wcastle(pos);
        if ((wc & 1) && !(F1G1 & c.allPieces) && !(F1G1 & c.threatened)) addMove(&l, 4, 6, FL_KING_CASTLE);
        if ((wc & 2) && !(B1D1 & c.allPieces) && !(C1D1 & c.threatened)) addMove(&l, 4, 2, FL_QUEEN_CASTLE);
    } else {
        int bc = st_bcastle(pos);
        if ((bc & 1) && !(F8G8 & c.allPieces) && !(F8G8 & c.threatened)) addMove(&l, 60, 62, FL_KING_CASTLE);
        if ((bc & 2) && !(B8D8 & c.allPieces) && !(C8D8 & c.threatened)) addMove(&l, 60, 58, FL_QUEEN_CASTLE);
    }
    return l.n;
}

/* ------------------------------------------------------------------- make */

/* updateCastleFlag, MoveGeneratorBitboard.h:1310-1340 (if/else form) */
static void updateCastleFlag(oracle_pos *pos, U64 dst, int chance)
{
    if (chance == WHITE) {
        int bc = st_bcastle(pos);
        if (dst & (U64)0x8000000000000000ULL) bc &= ~1;
        else if (dst & (U64)0x0100000000000000ULL) bc &= ~2;
        st_set_bcastle(pos, bc);
    } else {
        int wc = st_wcastle(pos);
        if (dst & (U64)0x80ULL) wc &= ~1;
        else if (dst & (U64)0x01ULL) wc &= ~2;
        st_set_wcastle(pos, wc);
    }
}

enum { PC_PAWN = 1, PC_KNIGHT, PC_BISHOP, PC_ROOK, PC_QUEEN, PC_KING };

/* makeMove without hash update, MoveGeneratorBitboard.h:3310-3570 */
void oracle_make_move(oracle_pos *pos, uint16_t move)
{
    int from = move & 63, to = (move >> 6) & 63, flags = move >> 12;
    int chance = st_chance(pos);
    U64 src = (U64)1 << from, dst = (U64)1 << to;
    U64 queens = (U64)pos->bb[P_BQ] & (U64)pos->bb[P_RQ];
    int piece;
    if ((U64)pos->bb[P_KINGS] & src) piece = PC_KING;
    else if ((U64)pos->bb[P_KNIGHTS] & src) piece = PC_KNIGHT;
    else if (((U64)pos->bb[P_PAWNS] & RANKS2TO7) & src) piece = PC_PAWN;
    else if (queens & src) piece = PC_QUEEN;
    else if ((U64)pos->bb[P_BQ] & src) piece = PC_BISHOP;
    else piece = PC_ROOK;

    if (flags == FL_PROMO_N || flags == FL_PROMO_N + 4) piece = PC_KNIGHT;
    else if (flags == FL_PROMO_B || flags == FL_PROMO_B + 4) piece = PC_BISHOP;
    else if (flags == FL_PROMO_R || flags == FL_PROMO_R + 4) piece = PC_ROOK;
    else if (flags == FL_PROMO_Q || flags == FL_PROMO_Q + 4) piece = PC_QUEEN;

    U64 pawnsState = (U64)pos->bb[P_PAWNS];
    U64 bq = (U64)pos->bb[P_BQ], rq = (U64)pos->bb[P_RQ], kings = (U64)pos->bb[P_KINGS];
    U64 knights = (U64)pos->bb[P_KNIGHTS], white = (U64)pos->bb[P_WHITE];

    bq &= ~src; rq &= ~src; kings &= ~src; knights &= ~src; pawnsState &= ~(src & RANKS2TO7);
    bq &= ~dst; rq &= ~dst; kings &= ~dst; knights &= ~dst; pawnsState &= ~(dst & RANKS2TO7);

    int wc = st_wcastle(pos), bc = st_bcastle(pos);
    if (piece == PC_KING) {
        kings |= dst;
        if (chance == WHITE) wc = 0; else bc = 0;
    }
    if (piece == PC_KNIGHT) knights |= dst;
    if (piece == PC_PAWN) pawnsState |= dst;
    if (piece == PC_BISHOP || piece == PC_QUEEN) bq |= dst;
    if (piece == PC_ROOK || piece == PC_QUEEN) rq |= dst;

    if (chance == WHITE) white = (white ^ src) | dst;
    else white = white & ~dst;

    if (flags == FL_EP_CAPTURE) {
        U64 cap = chance == WHITE ? southOne(dst) : northOne(dst);
        pawnsState &= ~(cap & RANKS2TO7);
        if (chance == BLACK) white &= ~cap;
    }
    if (chance == WHITE) {
        if (flags == FL_KING_CASTLE) { rq = (rq ^ (U64)0x80ULL) | (U64)0x20ULL; white = (white ^ (U64)0x80ULL) | (U64)0x20ULL; }
        else if (flags == FL_QUEEN_CASTLE) { rq = (rq ^ (U64)0x01ULL) | (U64)0x08ULL; white = (white ^ (U64)0x01ULL) | (U64)0x08ULL; }
    } else {
        if (flags == FL_KING_CASTLE) rq = (rq ^ (U64)0x8000000000000000ULL) | (U64)0x2000000000000000ULL;
        else if (flags == FL_QUEEN_CASTLE) rq = (rq ^ (U64)0x0100000000000000ULL) | (U64)0x0800000000000000ULL;
    }

    pos->bb[P_WHITE] = RAW(white);
    pos->bb[P_PAWNS] = RAW(pawnsState);
    pos->bb[P_KNIGHTS] = RAW(knights);
    pos->bb[P_BQ] = RAW(bq);
    pos->bb[P_RQ] = RAW(rq);
    pos->bb[P_KINGS] = RAW(kings);
    st_set_wcastle(pos, wc);
    st_set_bcastle(pos, bc);

    st_set_chance(pos, !chance);
    st_set_ep(pos, 0);
    updateCastleFlag(pos, dst, chance);
    if (piece == PC_ROOK) updateCastleFlag(pos, src, !chance);

    if (flags == FL_DOUBLE_PUSH) {
        /* EXACT_EN_PASSENT_FLAGGING (MoveGeneratorBitboard.h:3524-3541) */
        U64 allPawns = (U64)pos->bb[P_PAWNS] & RANKS2TO7;
        U64 allPieces = (U64)pos->bb[P_KINGS] | allPawns | (U64)pos->bb[P_KNIGHTS] |
                        (U64)pos->bb[P_BQ] | (U64)pos->bb[P_RQ];
        U64 blackPieces = allPieces & ~(U64)pos->bb[P_WHITE];
        U64 enemyPieces = chance == WHITE ? blackPieces : (U64)pos->bb[P_WHITE];
        U64 epSources = (eastOne(dst) | westOne(dst)) & allPawns & enemyPieces;
        if (epSources) st_set_ep(pos, (from & 7) + 1);
    }
}

/* ------------------------------------------------------------------ perft */

uint64_t oracle_perft(const oracle_pos *pos, uint32_t depth)
{
    if (depth == 0) return 1;
    if (depth == 1) return oracle_count_moves(pos);
    uint16_t moves[256];
    uint32_t n = oracle_generate_moves(pos, moves);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) {
        oracle_pos child = *pos;
        oracle_make_move(&child, moves[i]);
        total += oracle_perft(&child, depth - 1);
    }
    return total;
}

uint32_t oracle_divide(const oracle_pos *pos, uint32_t depth, uint16_t *moves, uint64_t *counts)
{
    uint32_t n = oracle_generate_moves(pos, moves);
    for (uint32_t i = 0; i < n; i++) {
        oracle_pos child = *pos;
        oracle_make_move(&child, moves[i]);
        counts[i] = depth >= 1 ? oracle_perft(&child, depth - 1) : 0;
    }
    return n;
}

/* ---------------------------------------------------------------- FEN */

/* Utils::readFENString (util.cpp:189-281) followed by board088ToHexBB
 * (util.cpp:92-140): board, side, castling letters, en-passant FILE only;
 * the half-move and full-move clocks are not read. */
int oracle_fen_to_pos(const char *fen, oracle_pos *out)
{
    oracle_init();
    memset(out, 0, sizeof(*out));
    int i = 0, row = 0, col = 0;
    for (; fen[i]; i++) {
        char ch = fen[i];
        if (ch == '/' || ch == '\\') {
            row++;
            col = 0;
        } else if (ch >= '1' && ch <= '8') {
            col += ch - '0';
        } else if (strchr("kqrbnpKQRBNP", ch)) {
            if (row > 7 || col > 7) return -1;
            int sq = (7 - row) * 8 + col;
            uint64_t bit = 1ULL << sq;
            if (ch >= 'A' && ch <= 'Z') out->bb[P_WHITE] |= bit;
            switch (ch | 0x20) {
            case 'p': out->bb[P_PAWNS] |= bit; break;
            case 'n': out->bb[P_KNIGHTS] |= bit; break;
            case 'b': out->bb[P_BQ] |= bit; break;
            case 'r': out->bb[P_RQ] |= bit; break;
            case 'q': out->bb[P_BQ] |= bit; out->bb[P_RQ] |= bit; break;
            case 'k': out->bb[P_KINGS] |= bit; break;
            }
            col++;
        } else if (ch == ' ') {
            break;
        }
        if (row >= 7 && col == 8) break;
    }
    if (!fen[i]) return -1;
    i++;
    while (fen[i] == ' ') i++;
    int chance = (fen[i] == 'b' || fen[i] == 'B') ? BLACK : WHITE;
    if (fen[i]) i++;
    while (fen[i] == ' ') i++;
    int wc = 0, bc = 0;
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
    int ep = 0;
    if (fen[i] >= 'a' && fen[i] <= 'h') ep = fen[i] - 'a' + 1;
    /* real pawns never stand on ranks 1/8; keep the state bits clean */
    out->bb[P_PAWNS] &= RANKS2TO7;
    st_set_chance(out, chance);
    st_set_wcastle(out, wc);
    st_set_bcastle(out, bc);
    st_set_ep(out, ep);
    if (popc((U64)(out->bb[P_KINGS] & out->bb[P_WHITE])) != 1 ||
        popc((U64)(out->bb[P_KINGS] & ~out->bb[P_WHITE])) != 1)
        return -1;
    return 0;
}

/* ---------------------------------------------------- threaded batch */

#ifndef ORACLE_OPCOUNT
typedef struct {
    oracle_pos pos;
    uint32_t depth, owner;
} otask;

typedef struct {
    otask *tasks;
    size_t ntasks;
    size_t *cursor;
    pthread_mutex_t *mu;
    uint64_t *partial; /* per-root sums for this worker */
} oworker;

static void *oworker_main(void *arg)
{
    oworker *w = (oworker *)arg;
    for (;;) {
        pthread_mutex_lock(w->mu);
        size_t i = (*w->cursor)++;
        pthread_mutex_unlock(w->mu);
        if (i >= w->ntasks) break;
        w->partial[w->tasks[i].owner] += oracle_perft(&w->tasks[i].pos, w->tasks[i].depth);
    }
    return NULL;
}

/* Root split: two plies expanded on the calling thread, subtrees pulled by
 * all workers from a shared cursor. */
int oracle_perft_batch_mt(const oracle_pos *pos, const uint32_t *depths, uint32_t n,
                          int threads, uint64_t *out)
{
    oracle_init();
    if (threads < 1) threads = 1;
    size_t cap = 1024, nt = 0;
    otask *tasks = (otask *)malloc(cap * sizeof(otask));
    if (!tasks) return -1;
    for (uint32_t r = 0; r < n; r++) {
        uint16_t m1[256], m2[256];
        if (depths[r] <= 3) {
            if (nt == cap) { cap *= 2; tasks = (otask *)realloc(tasks, cap * sizeof(otask)); }
            tasks[nt].pos = pos[r]; tasks[nt].depth = depths[r]; tasks[nt].owner = r; nt++;
            continue;
        }
        uint32_t n1 = oracle_generate_moves(&pos[r], m1);
        for (uint32_t i = 0; i < n1; i++) {
            oracle_pos c1 = pos[r];
            oracle_make_move(&c1, m1[i]);
            uint32_t n2 = oracle_generate_moves(&c1, m2);
            for (uint32_t j = 0; j < n2; j++) {
                if (nt == cap) { cap *= 2; tasks = (otask *)realloc(tasks, cap * sizeof(otask)); }
                tasks[nt].pos = c1;
                oracle_make_move(&tasks[nt].pos, m2[j]);
                tasks[nt].depth = depths[r] - 2;
                tasks[nt].owner = r;
                nt++;
            }
        }
    }
    size_t cursor = 0;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    oworker *ws = (oworker *)malloc(sizeof(oworker) * threads);
    for (int t = 0; t < threads; t++) {
        ws[t].tasks = tasks; ws[t].ntasks = nt; ws[t].cursor = &cursor; ws[t].mu = &mu;
        ws[t].partial = (uint64_t *)calloc(n, sizeof(uint64_t));
        pthread_create(&th[t], NULL, oworker_main, &ws[t]);
    }
    for (uint32_t r = 0; r < n; r++) out[r] = 0;
    for (int t = 0; t < threads; t++) {
        pthread_join(th[t], NULL);
        for (uint32_t r = 0; r < n; r++) out[r] += ws[t].partial[r];
        free(ws[t].partial);
    }
    free(ws);
    free(th);
    free(tasks);
    return 0;
}
#endif
