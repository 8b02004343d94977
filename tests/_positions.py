"""Crafted positions for edge cases that playouts rarely reach: many queens
behind a shielded king give 94-170 legal moves per node, the high end of
the move counts the level buffers and tile item tags must hold.  Each comes
with its colour mirror (black to move), which must count the same."""

MANY_MOVES = [
    "6nk/6pp/8/Q1Q1Q1Q1/8/Q1Q1Q1Q1/8/Q1Q1Q1QK w - - 0 1",
    "6nk/6pp/8/1Q1Q1Q1Q/8/Q1Q1Q1Q1/8/1Q1Q1Q1K w - - 0 1",
    "6rk/5npp/8/1Q1Q1Q2/8/Q1Q1Q1Q1/8/1Q1Q1Q1K w - - 0 1",
    "6rk/5bpp/Q7/2Q1Q1Q1/8/1Q1Q1Q2/8/Q1Q1Q2K w - - 0 1",
]


def mirror_fen(fen: str) -> str:
    """Colour mirror: ranks reversed, colours swapped, the other side to
    move; castling letters swap case and the en-passant rank flips."""
    parts = fen.split()
    board = "/".join(r.swapcase() for r in reversed(parts[0].split("/")))
    side = "b" if parts[1] == "w" else "w"
    castle = parts[2] if parts[2] == "-" else "".join(sorted(parts[2].swapcase(), key="KQkq".index))
    ep = parts[3] if parts[3] == "-" else parts[3][0] + ("6" if parts[3][1] == "3" else "3")
    return " ".join([board, side, castle, ep] + parts[4:])


def many_moves_with_mirrors():
    return [f for fen in MANY_MOVES for f in (fen, mirror_fen(fen))]
