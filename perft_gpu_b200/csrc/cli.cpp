// Command-line front end over the C ABI (include/perft_b200.h).
//
//   perft_gpu <fen|startpos> <depth> [<gpus>] [<launchdepth>]
//       The reference's process CLI (perft.cu:14-164): prints Perft(NN) for
//       every depth from 3 (or depth, if smaller) up to <depth>, each with
//       its wall time.  Above depth 10 the root moves' subtotals are printed
//       first, as the reference's divided perft does (launcher.h:1344-1351),
//       computed by the host root split with transposition merging.  With
//       <gpus> above 1 those deep counts are split over that many GPUs (the
//       reference's one host thread per GPU, launcher.h:409-583): one shard
//       process per GPU (GPU i runs perft_deep_shard shard i of <gpus>), and
//       the per-move subtotals are summed here.  Shallower depths run on one
//       GPU (PERFT_DEVICE).  <launchdepth> is accepted and ignored: level
//       sizes are planned from measured counts.
//       With PERFT_STORE=<file> the subtrees finished by a deep run are kept
//       in that file, and a stopped run started again skips them.
//       PERFT_DIVIDED_DEPTH moves the divided threshold (default 10).
//   perft_gpu --records <file> [<depth>]
//       Records mode (launcher.h:1579-1695): "<line> <perft> <perft*count>"
//       per input line appended to <file>.op, resuming after the lines
//       already written.  Depth defaults to 7.
//   perft_gpu --uci
//       A minimal UCI loop (uci, isready, ucinewgame, position startpos|fen
//       ... [moves ...], go perft N, d, quit).  The reference's UCI is a stub
//       (UciInterface.cpp:7); "go perft" prints one "move: count" line per
//       root move, then "Nodes searched: N".
#include <chrono>
#include <map>
#include <signal.h>
#include <stdio.h>
#include <sys/wait.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>

#include "../../include/perft_b200.h"

namespace {

const char *START_FEN = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1";
bool g_ready = false;

int ensure_init()
{
    if (g_ready) return PERFT_OK;
    perft_config cfg;
    perft_config_default(&cfg);
    if (const char *d = getenv("PERFT_DEVICE")) cfg.device = atoi(d);
    if (const char *a = getenv("PERFT_ARENA_GB")) cfg.arena_bytes = (uint64_t)(atof(a) * (1ull << 30));
    if (const char *t = getenv("PERFT_TT_LOG2")) cfg.tt_log2_entries = (uint32_t)atoi(t);
    if (const char *z = getenv("PERFT_ZOBRIST_SEED")) cfg.zobrist_seed = strtoull(z, nullptr, 0);
    const int rc = perft_init(&cfg);
    if (rc != PERFT_OK) {
        fprintf(stderr, "perft_init failed: %s\n", perft_status_string(rc));
        return rc;
    }
    if (const char *st = getenv("PERFT_STORE")) {
        const int src = perft_result_store_open(st);
        if (src != PERFT_OK) {
            fprintf(stderr, "cannot open result store %s: %s\n", st, perft_status_string(src));
            perft_shutdown();
            return src;
        }
    }
    g_ready = true;
    return PERFT_OK;
}

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void usage()
{
    printf("Usage perft_gpu <fen> <depth> [<gpus>] [<launchdepth>]\n"
           "      perft_gpu --records <file> [<depth>]\n"
           "      perft_gpu --uci\n");
}

typedef unsigned __int128 u128;

// Depths above this print divided output through the deep path (the
// reference's DIVIDED_PERFT_DEPTH, launcher.h:21); PERFT_DIVIDED_DEPTH
// overrides it.
int divided_from()
{
    const char *e = getenv("PERFT_DIVIDED_DEPTH");
    return e ? atoi(e) : 10;
}

// Host split of a deep count: the frontier sits 1 + split plies below the
// root, at most five (about 10^6 distinct boards from the initial position).
uint32_t split_for(uint32_t depth)
{
    uint32_t s = depth > 8 ? depth - 7 : 1;
    if (s > 4) s = 4;
    return s + 1 > depth ? depth - 1 : s;
}

// Decimal digits of a 128-bit count (totals beyond 64 bits: perft 14+).
std::string to_dec(u128 v)
{
    std::string s;
    do {
        s.insert(s.begin(), (char)('0' + (int)(v % 10)));
        v /= 10;
    } while (v);
    return s;
}

// Deep divided count split over `gpus` shard processes: this program is
// re-executed as "--deep-shard <i> <n> <depth> <split> <fen>" once per GPU
// (a fresh process each, so every one initialises CUDA itself), each prints
// "<move> <subtotal>" lines and "END", and the subtotals are summed here.
int divided_sharded(const std::string &fen, uint32_t depth, uint32_t split, int gpus, std::vector<std::string> &moves,
                    std::vector<uint64_t> &counts, u128 *total)
{
    std::vector<pid_t> pids;
    std::vector<FILE *> outs;
    const std::string dep = std::to_string(depth), spl = std::to_string(split), n = std::to_string(gpus);
    // a failed start stops and reaps the shards already running
    auto abandon = [&]() {
        for (FILE *f : outs)
            if (f) fclose(f);
        for (pid_t pid : pids) kill(pid, SIGTERM);
        for (pid_t pid : pids) waitpid(pid, nullptr, 0);
        return PERFT_ERR_INTERNAL;
    };
    for (int i = 0; i < gpus; i++) {
        int fd[2];
        if (pipe(fd) != 0) return abandon();
        const pid_t pid = fork();
        if (pid < 0) {
            close(fd[0]);
            close(fd[1]);
            return abandon();
        }
        if (pid == 0) {
            dup2(fd[1], 1);
            close(fd[0]);
            close(fd[1]);
            const std::string si = std::to_string(i);
            execl("/proc/self/exe", "perft_gpu", "--deep-shard", si.c_str(), n.c_str(), dep.c_str(), spl.c_str(),
                  fen.c_str(), (char *)nullptr);
            _exit(127);
        }
        close(fd[1]);
        pids.push_back(pid);
        outs.push_back(fdopen(fd[0], "r"));
    }
    std::map<std::string, uint64_t> sum;
    std::vector<std::string> order;
    bool ok = true;
    for (size_t i = 0; i < outs.size(); i++) {
        char line[256];
        bool ended = false;
        while (outs[i] && fgets(line, sizeof line, outs[i])) {
            char mv[16];
            unsigned long long c = 0;
            if (!strncmp(line, "END", 3)) {
                ended = true;
                break;
            }
            if (sscanf(line, "%15s %llu", mv, &c) != 2) continue;
            if (!sum.count(mv)) order.push_back(mv);
            sum[mv] += c;
        }
        if (outs[i]) fclose(outs[i]);
        ok = ok && ended;
    }
    for (pid_t pid : pids) {
        int st = 0;
        if (waitpid(pid, &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) ok = false;
    }
    if (!ok) return PERFT_ERR_INTERNAL;
    moves.clear();
    counts.clear();
    *total = 0;
    for (const std::string &m : order) {
        moves.push_back(m);
        counts.push_back(sum[m]);
        *total += sum[m];
    }
    return PERFT_OK;
}

// One shard of a deep divided count (the child side of divided_sharded):
// device = shard index unless PERFT_SHARD_DEVICE pins every shard to one GPU.
int run_deep_shard(int argc, char **argv)
{
    if (argc < 7) return 2;
    const uint32_t shard = (uint32_t)atoi(argv[2]), n = (uint32_t)atoi(argv[3]);
    const uint32_t depth = (uint32_t)atoi(argv[4]), split = (uint32_t)atoi(argv[5]);
    perft_pos48 pos;
    if (perft_fen_to_pos(argv[6], &pos) != PERFT_OK) return 2;
    if (!getenv("PERFT_SHARD_DEVICE")) {
        char dev[16];
        snprintf(dev, sizeof dev, "%u", shard);
        setenv("PERFT_DEVICE", dev, 1);
    } else {
        setenv("PERFT_DEVICE", getenv("PERFT_SHARD_DEVICE"), 1);
    }
    if (ensure_init() != PERFT_OK) return 1;
    char mv[256][6];
    uint64_t c[256], t = 0;
    uint32_t nm = 0;
    const int rc = perft_deep_shard(&pos, depth, split, shard, n, mv, c, &nm, &t);
    if (rc != PERFT_OK && !(rc == PERFT_ERR_OVERFLOW && nm > 0)) {
        fprintf(stderr, "shard %u failed: %s\n", shard, perft_status_string(rc));
        return 1;
    }
    for (uint32_t i = 0; i < nm; i++) printf("%s %llu\n", mv[i], (unsigned long long)c[i]);
    printf("END\n");
    return 0;
}

// Divided count of pos at depth: one subtotal per root move, summed in 128
// bits (the engine reports PERFT_ERR_OVERFLOW when only the total exceeds 64
// bits, with the subtotals filled in).
int divided(const perft_pos48 &pos, uint32_t depth, std::vector<std::string> &moves,
            std::vector<uint64_t> &counts, u128 *total)
{
    char mv[256][6];
    uint64_t c[256];
    uint32_t n = 0;
    uint64_t t64 = 0;
    int rc;
    if (depth > divided_from()) {
        rc = perft_deep(&pos, depth, split_for(depth), mv, c, &n, &t64);
    } else {
        rc = perft_divide(&pos, depth, mv, c, &n);
    }
    if (rc != PERFT_OK && !(rc == PERFT_ERR_OVERFLOW && n > 0)) return rc;
    moves.clear();
    counts.clear();
    *total = 0;
    for (uint32_t i = 0; i < n; i++) {
        moves.emplace_back(mv[i]);
        counts.push_back(c[i]);
        *total += c[i];
    }
    return PERFT_OK;
}

int run_cli(int argc, char **argv)
{
    std::string fen = argv[1];
    if (fen == "startpos" || fen.size() <= 5) fen = START_FEN;
    const int maxDepth = atoi(argv[2]);
    const int gpus = argc >= 4 ? atoi(argv[3]) : 1;
    if (maxDepth < 0 || maxDepth > 30 || gpus < 1 || gpus > 64) {
        usage();
        return 2;
    }
    perft_pos48 pos;
    int rc = perft_fen_to_pos(fen.c_str(), &pos);
    if (rc != PERFT_OK) {
        fprintf(stderr, "bad FEN: %s\n", perft_status_string(rc));
        return 2;
    }
    if (!(gpus > 1 && (maxDepth < 3 ? maxDepth : 3) > divided_from()) && (rc = ensure_init()) != PERFT_OK) return 1;
    char canon[128];
    perft_pos_to_fen(&pos, canon, sizeof canon);
    printf("%s\n", canon);
    const int minDepth = maxDepth < 3 ? maxDepth : 3;
    for (int d = minDepth; d <= maxDepth; d++) {
        const double t0 = now_s();
        u128 total = 0;
        if (d > divided_from()) {
            std::vector<std::string> mv;
            std::vector<uint64_t> c;
            if (gpus > 1 && g_ready) {
                perft_shutdown();  // the shard processes take the GPUs (and their memory) from here on
                g_ready = false;
            }
            rc = gpus > 1 ? divided_sharded(fen, (uint32_t)d, split_for((uint32_t)d), gpus, mv, c, &total)
                          : divided(pos, (uint32_t)d, mv, c, &total);
            if (rc == PERFT_OK)
                for (size_t i = 0; i < mv.size(); i++) printf("%s   %20llu\n", mv[i].c_str(), (unsigned long long)c[i]);
        } else {
            uint64_t t64 = 0;
            if (!g_ready && (rc = ensure_init()) != PERFT_OK) return 1;
            rc = perft(&pos, (uint32_t)d, &t64);
            total = t64;
        }
        if (rc != PERFT_OK) {
            fprintf(stderr, "perft(%d) failed: %s\n", d, perft_status_string(rc));
            return 1;
        }
        printf("Perft(%02d):%20s, time: %8g s\n", d, to_dec(total).c_str(), now_s() - t0);
        fflush(stdout);
    }
    return 0;
}

int run_records(int argc, char **argv)
{
    if (argc < 3) {
        usage();
        return 2;
    }
    const uint32_t depth = argc >= 4 ? (uint32_t)atoi(argv[3]) : 7;
    if (ensure_init() != PERFT_OK) return 1;
    printf("filename of op: %s.op\n", argv[2]);
    const double t0 = now_s();
    uint64_t done = 0;
    const int rc = perft_records(argv[2], depth, 0, &done);
    if (rc != PERFT_OK) {
        fprintf(stderr, "records failed: %s\n", perft_status_string(rc));
        return 1;
    }
    const double t = now_s() - t0;
    printf("Records done: %llu, Total: %g seconds, Avg: %g seconds\n", (unsigned long long)done, t,
           done ? t / (double)done : 0.0);
    return 0;
}

// Splits a line into whitespace-separated tokens.
std::vector<std::string> tokens(const char *line)
{
    std::vector<std::string> out;
    std::string cur;
    for (const char *p = line; *p; p++) {
        if (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += *p;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

int run_uci()
{
    perft_pos48 pos;
    perft_fen_to_pos(START_FEN, &pos);
    char line[8192];
    while (fgets(line, sizeof line, stdin)) {
        const std::vector<std::string> t = tokens(line);
        if (t.empty()) continue;
        const std::string &cmd = t[0];
        if (cmd == "quit") {
            break;
        } else if (cmd == "uci") {
            printf("id name perft_gpu_b200\nid author perft_gpu_b200 contributors\nuciok\n");
        } else if (cmd == "isready") {
            printf("readyok\n");
        } else if (cmd == "ucinewgame") {
            perft_fen_to_pos(START_FEN, &pos);
        } else if (cmd == "position" && t.size() >= 2) {
            size_t i = 1;
            std::string fen;
            if (t[1] == "startpos") {
                fen = START_FEN;
                i = 2;
            } else if (t[1] == "fen") {
                for (i = 2; i < t.size() && t[i] != "moves"; i++) fen += (fen.empty() ? "" : " ") + t[i];
            }
            perft_pos48 p;
            if (perft_fen_to_pos(fen.c_str(), &p) != PERFT_OK) {
                printf("info string bad fen\n");
                fflush(stdout);
                continue;
            }
            bool ok = true;
            if (i < t.size() && t[i] == "moves")
                for (i++; i < t.size() && ok; i++) ok = perft_apply_uci_move(&p, t[i].c_str()) == PERFT_OK;
            if (!ok)
                printf("info string illegal move %s\n", t[i - 1].c_str());
            else
                pos = p;
        } else if (cmd == "d") {
            char fen[128];
            perft_pos_to_fen(&pos, fen, sizeof fen);
            printf("Fen: %s\n", fen);
        } else if (cmd == "go" && t.size() >= 3 && t[1] == "perft") {
            const int depth = atoi(t[2].c_str());
            if (depth < 1 || depth > 30) {
                printf("info string bad depth\n");
            } else if (ensure_init() == PERFT_OK) {
                std::vector<std::string> mv;
                std::vector<uint64_t> c;
                u128 total = 0;
                const double t0 = now_s();
                const int rc = divided(pos, (uint32_t)depth, mv, c, &total);
                if (rc != PERFT_OK) {
                    printf("info string perft failed: %s\n", perft_status_string(rc));
                } else {
                    for (size_t k = 0; k < mv.size(); k++) printf("%s: %llu\n", mv[k].c_str(), (unsigned long long)c[k]);
                    const double dt = now_s() - t0;
                    printf("\nNodes searched: %s\ninfo string time %g s, %g leaves/s\n\n", to_dec(total).c_str(), dt,
                           dt > 0 ? (double)total / dt : 0.0);
                }
            } else {
                printf("info string no GPU engine\n");
            }
        } else {
            printf("info string unknown command %s\n", cmd.c_str());
        }
        fflush(stdout);
    }
    if (g_ready) perft_shutdown();
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc >= 2 && (!strcmp(argv[1], "--help") || !strcmp(argv[1], "-h"))) {
        usage();
        return 0;
    }
    if (argc >= 2 && !strcmp(argv[1], "--uci")) return run_uci();
    if (argc >= 2 && !strcmp(argv[1], "--records")) return run_records(argc, argv);
    if (argc >= 2 && !strcmp(argv[1], "--deep-shard")) {
        const int rc = run_deep_shard(argc, argv);
        if (g_ready) perft_shutdown();
        return rc;
    }
    if (argc < 3) {
        usage();
        printf("\nAs no parameters were provided... running the start position to depth 5\n");
        static char a0[] = "perft_gpu", a1[] = "startpos", a2[] = "5";
        char *def[] = {a0, a1, a2};
        const int rc = run_cli(3, def);
        if (g_ready) perft_shutdown();
        return rc;
    }
    const int rc = run_cli(argc, argv);
    if (g_ready) perft_shutdown();
    return rc;
}
