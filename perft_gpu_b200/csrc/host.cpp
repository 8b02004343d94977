// Host-side utilities of the C ABI: FEN parsing and printing, UCI move
// strings, divided perft, seeded playout positions.  They use the host build
// of the move generator for move lists only; every leaf count is computed by
// the GPU engine (engine.cu).
#include <random>
#include <string>
#include <vector>

#include <stdio.h>
#include <string.h>

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

int perft_divide(const perft_pos48 *pos, uint32_t depth, char (*moves)[6], uint64_t *counts,
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

}  // extern "C"
