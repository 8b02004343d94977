/*
 * perft_b200 — C ABI of the B200 perft engine.
 *
 * Drop-in boundary for the perft path of ankan-ban/perft_gpu.  The reference
 * exposes no library: its entry points are internal C++ functions behind the
 * `perft_gpu <fen> <depth>` command line (perft.cu:14-164).  Each function
 * below replaces one of them; the citation names the reference routine.
 *
 * Positions use the reference's 48-byte HexaBitBoardPosition layout
 * (chess.h:208-230), so a caller holding reference positions passes them
 * unchanged.  Counts are exact uint64 leaf counts.  Every entry point returns
 * a status code (PERFT_OK or a negative PERFT_ERR_*) instead of the
 * reference's printf/exit(0) and ALLSET sentinel (perft_bb.h:1360,1499).
 *
 * The entry points are thread-safe: calls on one process-wide engine are
 * serialised by an internal lock.  All perft computation runs on the GPU;
 * there is no CPU fallback — without a usable CUDA device, perft_init fails
 * with PERFT_ERR_NO_DEVICE.
 */
#ifndef PERFT_B200_H
#define PERFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define PERFT_OK                   0
#define PERFT_PENDING              1  /* serving: the query is still running */
#define PERFT_ERR_INVALID_ARG     -1
#define PERFT_ERR_NOT_INITIALIZED -2
#define PERFT_ERR_CUDA            -3
#define PERFT_ERR_OUT_OF_MEMORY   -4  /* replaces the reference's ALLSET sentinel */
#define PERFT_ERR_INTERNAL        -5  /* a device-side consistency check failed */
#define PERFT_ERR_BAD_FEN         -6
#define PERFT_ERR_NO_DEVICE       -7
#define PERFT_ERR_ILLEGAL_MOVE    -8
#define PERFT_ERR_TIMEOUT         -9
#define PERFT_ERR_NOT_FOUND      -10
#define PERFT_ERR_IO             -11
#define PERFT_ERR_OVERFLOW       -12  /* a count does not fit 64 bits (the reference's InfInt range) */

/* ---------------------------------------------------------------- types */

/* Byte-compatible with HexaBitBoardPosition (chess.h:208-230):
 * bb[0] white pieces, bb[1] pawns with packed state (bits 0-1 white
 * castling, 2-3 black castling, 4-7 en-passant file + 1, 63 side to move),
 * bb[2] knights, bb[3] bishops|queens, bb[4] rooks|queens, bb[5] kings. */
typedef struct perft_pos48 {
    uint64_t bb[6];
} perft_pos48;

/* Slider attack implementation (the reference's USE_SLIDING_LUT switch,
 * switches.h:108-125, made a run-time choice). */
#define PERFT_SLIDERS_AUTO      -1  /* autotuned per ply kind at init */
#define PERFT_SLIDERS_KOGGE      0  /* Kogge-Stone occluded fills */
#define PERFT_SLIDERS_MAGIC      1  /* fancy magic lookups */
#define PERFT_SLIDERS_KOGGE_FMA  2  /* Kogge-Stone, constant shifts on the FMA pipe */
#define PERFT_SLIDERS_KOGGE_SPLIT 3 /* Kogge-Stone, left shifts split over ALU and FMA pipes */
#define PERFT_SLIDERS_HYBRID      4 /* attack map by fills, own slider moves by magic lookups */

typedef struct perft_config {
    int      device;          /* CUDA device ordinal */
    uint64_t arena_bytes;     /* level-buffer budget in HBM; 0 = 85% of free */
    int      sliders_expand;  /* PERFT_SLIDERS_* for interior plies */
    int      sliders_leaf;    /* PERFT_SLIDERS_* for the count-only last ply */
    int      tt_log2_entries; /* transposition table size; 0 = no table */
    uint64_t zobrist_seed;    /* seed of the two sets of 781 Zobrist keys (TT only) */
} perft_config;

/* Defaults: device 0, automatic arena, autotuned sliders, no TT. */
void perft_config_default(perft_config *cfg);

/* Engine set-up: allocates the arena, uploads move-generator tables,
 * autotunes.  Replaces initGPU + MoveGeneratorBitboard::init
 * (launcher.h:1506-1533, MoveGeneratorBitboard.h:982-1201). */
int perft_init(const perft_config *cfg);
int perft_shutdown(void);
const char *perft_status_string(int status);

/* Leaf count of one position: perft_bb / perftLauncher
 * (perft_bb.h:79-101, launcher.h:1455-1503), returned instead of printed.
 * The count must fit 64 bits (up to perft 13 of the initial position);
 * perft_deep reports larger totals through exact per-move subtotals. */
int perft(const perft_pos48 *pos, uint32_t depth, uint64_t *out);

/* Batched perft: out[i] = perft(pos[i], depths[i]).  Host buffers.
 * Replaces the batch form of perft_bb_gpu_simple_hash (perft_bb.h:1242)
 * used by perft_bb_last_level_launcher (launcher.h:966-1143) and the
 * perft-records mode (launcher.h:1579-1695). */
int perft_batch(const perft_pos48 *pos, const uint8_t *depths, uint32_t n, uint64_t *out);

/* Same with positions and results already in device memory (depths stay on
 * the host: they drive the launch plan).  Synchronous. */
int perft_batch_device(const perft_pos48 *d_pos, const uint8_t *depths, uint32_t n,
                       uint64_t *d_out);

/* Divided perft: the legal moves of pos (UCI strings, 6 bytes each incl.
 * NUL) and the perft(depth-1) of each child.  Replaces dividedPerft's
 * per-move subtotals (launcher.h:1392-1450, 456-464). */
int perft_divide(const perft_pos48 *pos, uint32_t depth, char (*moves)[6], uint64_t *counts,
                 uint32_t *n_moves);

/* Allocation-free batched perft.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: processes whose HBM is
 * already reserved by another allocator (a serving framework, torch's
 * caching allocator), and latency-critical callers that cannot afford
 * cudaMalloc's implicit device-wide synchronisation.  Same contract as
 * perft_batch_device (device positions and results, host depths), plus the
 * caller's stream (NULL = legacy default stream); needs no perft_init and
 * allocates nothing: all working memory is one scratch array of
 * PERFT_NOALLOC_SCRATCH_BYTES compiled into the library, which every GPU
 * that loads the library keeps until the process exits.  Batches whose
 * levels do not fit it fail with PERFT_ERR_OUT_OF_MEMORY (use the arena
 * entry points for those).  All calls share the scratch, which keeps the
 * last call's contents (each call clears what must start at zero); calls
 * whose GPU work overlapped would race on it, so calls are serialised by a
 * lock, and every call, a failing one included, waits for its stream before
 * it returns: the call is synchronous.  The first call on a device does the
 * set-up (uploads the move tables, looks up the scratch address with that
 * device current).  Later calls look the address up again and redo the
 * set-up if the device's context was re-created (cudaDeviceReset). */
#define PERFT_NOALLOC_SCRATCH_BYTES (32ull << 20)
int perft_batch_noalloc(const perft_pos48 *d_pos, const uint8_t *depths, uint32_t n,
                        uint64_t *d_out, void *stream);

/* ------------------------------------------------------------- serving
 * Continuous batching of perft queries (no counterpart in the reference,
 * which runs one perft at a time from its CLI).  Queries of mixed depth are
 * submitted at any time; admitted queries keep their frontier levels in
 * HBM, and the levels of all in-flight queries with the same remaining
 * depth are advanced together, a bounded number of items per scheduler
 * iteration.  A query is admitted when its predicted level-buffer memory
 * fits the budget.  Counts are identical to perft(). */
typedef struct perft_serve_config {
    uint64_t memory_bytes;   /* budget for resident frontiers (0: 90% of the free arena) */
    uint64_t step_items;     /* items a level may advance per iteration (0: 2^27) */
    uint32_t max_in_flight;  /* admitted queries at once (0: 4096, at most 65536) */
    int32_t  use_tt;         /* 1 (default): frontier levels two and three plies above the leaves
                                probe, de-duplicate and store into the engine's transposition table
                                (perft_init with tt_log2_entries > 0), shared by every query
                                and kept across queries; 0: no table */
} perft_serve_config;

typedef struct perft_serve_stats {
    uint64_t submitted, completed, in_flight, queued;
    uint64_t iterations, launches;
    uint64_t memory_budget, memory_reserved, memory_peak;
    int      last_error;
    /* table use by the server since perft_serve_start: nodes probed, answered
     * from the table, merged with an identical node of the same level, stored */
    uint64_t tt_probes, tt_hits, tt_merged, tt_stores;
} perft_serve_stats;

void perft_serve_config_default(perft_serve_config *cfg);
int perft_serve_start(const perft_serve_config *cfg);   /* after perft_init */
int perft_serve_stop(void);
int perft_serve_submit(const perft_pos48 *pos, uint32_t depth, uint64_t *ticket);
/* PERFT_OK with the count (and submit-to-completion latency) once done,
 * PERFT_PENDING while running, PERFT_ERR_NOT_FOUND for unknown tickets.
 * A completed ticket is consumed by the call that returns it. */
int perft_serve_poll(uint64_t ticket, uint64_t *count, double *latency_s);
int perft_serve_wait(uint64_t ticket, double timeout_s, uint64_t *count, double *latency_s);
int perft_serve_get_stats(perft_serve_stats *out);

/* Deep perft by host root split (perft 11+): for every legal root move the
 * distinct positions split_plies below it are merged with their path counts
 * (a host transposition merge, like the reference's complete TT,
 * launcher.h:585-697) and searched on the GPU at the remaining depth.
 * moves/counts (optional, 256 entries) receive the per-move subtotals, the
 * divided perft of launcher.h:1344-1351.  Counts are 64-bit: when the total
 * does not fit (the reference switches to InfInt there), PERFT_ERR_OVERFLOW
 * is returned with every per-move subtotal filled in, to be summed wider by
 * the caller; a subtotal that does not fit fails the call with the same
 * status and *n_moves = 0. */
int perft_deep(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, char (*moves)[6],
               uint64_t *counts, uint32_t *n_moves, uint64_t *total);
/* One shard of perft_deep: only frontier boards i with i % n_shards == shard
 * are searched.  The frontier order is deterministic, so the per-move
 * subtotals of shards 0..n_shards-1 (one process per GPU) sum to perft_deep's:
 * the multi-GPU root split of launcher.h:476-583 with one 8-byte-per-move sum
 * as the only exchange. */
int perft_deep_shard(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint32_t shard,
                     uint32_t n_shards, char (*moves)[6], uint64_t *counts, uint32_t *n_moves,
                     uint64_t *total);

/* Size of the frontier perft_deep(pos, depth, split_plies) would search:
 * distinct boards and the move paths reaching them (host only, no GPU), for
 * choosing split_plies.  No counterpart in the reference. */
int perft_deep_frontier(const perft_pos48 *pos, uint32_t depth, uint32_t split_plies, uint64_t *n_boards,
                        uint64_t *n_paths);

/* Result store for deep runs: the counts of completed frontier subtrees,
 * keyed by the exact board and remaining depth.  perft_deep / perft_deep_shard
 * look every frontier board up before searching it and add what they search.
 * With a path, every completed GPU batch is appended to that file (64-byte
 * checksummed records after a 64-byte header) and flushed, so a run that is
 * stopped and started again with the same file skips the finished subtrees:
 * the checkpoint/resume role of the reference's disk hash (launcher.h:699-790,
 * perfthash.dat).  A torn last record is dropped on open.  A NULL path keeps
 * the store in host memory only (the reference's complete TT,
 * launcher.h:585-697). */
int perft_result_store_open(const char *path);
int perft_result_store_close(void);
int perft_result_store_stats(uint64_t *entries, uint64_t *hits, uint64_t *appended);

/* Records mode (launcher.h:1579-1695): each line of in_path is a FEN ending
 * with an occurrence count; "<line> <perft> <perft*count>" is appended to
 * in_path.op.  Lines already in the output are skipped (resume): the k-th
 * complete output line belongs to the k-th non-empty input line (empty
 * lines are neither searched nor counted); a torn last output line, left by
 * a run stopped in the middle of a write, is cut off and its record searched
 * again.  Input lines are read up to 2047 characters.  batch 0 means 4096
 * records per GPU batch.  PERFT_ERR_IO: the output cannot be read, opened
 * or written. */
int perft_records(const char *in_path, uint32_t depth, uint32_t batch, uint64_t *records_done);

/* ------------------------------------------------------- host utilities */

/* FEN -> position: Utils::readFENString + board088ToHexBB
 * (util.cpp:189-281, util.cpp:92-140).  Clocks are ignored; the en-passant
 * square contributes its file only. */
int perft_fen_to_pos(const char *fen, perft_pos48 *out);
int perft_pos_to_fen(const perft_pos48 *pos, char *buf, size_t len);

/* Legal moves in UCI notation, space separated (host move generator). */
int perft_legal_moves_uci(const perft_pos48 *pos, char *buf, size_t len, uint32_t *n_moves);
/* Applies one legal UCI move ("e2e4", "e7e8q"). */
int perft_apply_uci_move(perft_pos48 *pos, const char *uci);

/* Seeded random legal playouts from the initial position (std::mt19937_64,
 * uniform move choice), rejecting positions without legal moves. */
int perft_random_playouts(uint64_t seed, uint32_t n, uint32_t min_plies, uint32_t max_plies,
                          perft_pos48 *out);

/* Feature bits used to stratify synthetic workloads: 1 a legal en-passant
 * capture exists, 2 the side to move has a pawn on its 7th rank, 4 a
 * castling right remains, 8 the side to move is in check, 16 a promotion
 * move exists. */
int perft_position_features(const perft_pos48 *pos, uint32_t *features);

/* ------------------------------------------------------------- statistics */
typedef struct perft_stats {
    uint64_t leaf_launches;      /* count-only tile kernel launches */
    uint64_t expand_launches;    /* interior tile kernel launches */
    uint64_t other_launches;     /* scan / init kernels */
    uint64_t leaf_items;         /* (parent, move) pairs counted by leaf kernels */
    uint64_t leaf_parents;       /* parents whose moves the leaf kernels generated */
    uint64_t expand_items;       /* children written by interior kernels */
    double   leaf_ms;            /* CUDA-event time of leaf kernels */
    double   expand_ms;          /* CUDA-event time of interior kernels */
    int      sliders_expand;     /* variant in use */
    int      sliders_leaf;
    uint64_t arena_bytes;
    uint64_t peak_arena_bytes;
    uint32_t chunked_levels;     /* levels split to fit the arena */
    uint64_t tt_entries;         /* transposition-table size (0: no table) */
    uint64_t tt_probes;          /* nodes looked up */
    uint64_t tt_hits;            /* lookups answered by the table */
    uint64_t tt_duplicates;      /* same-level transpositions expanded once */
    uint64_t tt_stores;          /* entries written */
    uint64_t graph_launches;     /* batches run as one replayed device-driven graph */
    uint64_t small_launches;     /* single positions of depth 2..5 counted in one launch */
} perft_stats;

int perft_get_stats(perft_stats *out);

/* Launch configuration in use per (ply kind, remaining depth): chosen by the
 * per-depth autotuner at perft_init when the sliders are PERFT_SLIDERS_AUTO,
 * else the configured variant with the largest tiles.  Entries: the
 * count-only ply (remaining depth 2), then interior plies by remaining depth
 * 3..N (deeper plies use entry N).  No counterpart in the reference, whose
 * launch shape is fixed at compile time (switches.h:13-26). */
typedef struct perft_tune_entry {
    int    leaf;         /* 1: count-only last ply; 0: interior ply */
    int    remaining;    /* remaining depth of the parent level */
    int    sliders;      /* PERFT_SLIDERS_* variant */
    int    tile_log2;    /* largest tile (log2 items); small levels use smaller tiles */
    int    ctas_per_sm;  /* resident CTAs per SM; 0: all that fit */
    double calib_ms;     /* median calibration time of this key; 0: not timed */
} perft_tune_entry;
int perft_get_tuning(perft_tune_entry *out, uint32_t cap, uint32_t *n);
int perft_reset_stats(void);

/* Empties the transposition table (entries stay valid across calls, since a
 * position's perft never changes; clearing only matters for timing). */
int perft_tt_clear(void);

#ifdef __cplusplus
}
#endif

#endif /* PERFT_B200_H */
