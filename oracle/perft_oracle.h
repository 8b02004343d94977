/* Test infrastructure: CPU oracle for perft (clean-room restatement of the
 * reference host move generator).  Only tests/, the smoke check and bench.py's
 * CPU-baseline leg may load this; it is the checker, never the product.
 *
 * Position layout is byte-compatible with the reference's HexaBitBoardPosition
 * (chess.h:208-230): six uint64 bitboards
 *   [0] white pieces  [1] pawns (+ packed state)  [2] knights
 *   [3] bishops|queens  [4] rooks|queens  [5] kings
 * with the state packed into the pawn board's rank-1 and rank-8 bytes:
 *   bits 0-1 white castle (1 = king side, 2 = queen side), bits 2-3 black
 *   castle, bits 4-7 en-passant file + 1, bits 56-62 half-move counter,
 *   bit 63 side to move (0 white, 1 black).
 *
 * Moves are 16-bit: from (bits 0-5), to (6-11), flags (12-15) with the
 * reference's CMove flag codes (chess.h:234-293).
 */
#ifndef PERFT_ORACLE_H
#define PERFT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_pos {
    uint64_t bb[6];
} oracle_pos;

int      oracle_init(void);
int      oracle_fen_to_pos(const char *fen, oracle_pos *out);
uint32_t oracle_count_moves(const oracle_pos *pos);
uint32_t oracle_generate_moves(const oracle_pos *pos, uint16_t *moves);
void     oracle_make_move(oracle_pos *pos, uint16_t move);
uint64_t oracle_perft(const oracle_pos *pos, uint32_t depth);
uint32_t oracle_divide(const oracle_pos *pos, uint32_t depth, uint16_t *moves, uint64_t *counts);
int      oracle_perft_batch_mt(const oracle_pos *pos, const uint32_t *depths, uint32_t n,
                               int threads, uint64_t *out);

#ifdef __cplusplus
}
#endif

#endif
