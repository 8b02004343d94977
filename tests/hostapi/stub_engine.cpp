// Test-only: the host side of the C ABI (perft_gpu_b200/csrc/host.cpp:
// divided and deep perft, shards, the result store, records mode, FEN and
// move utilities) linked against a stand-in for the GPU engine that counts
// with the product's move generator compiled for the host.  The CPU test
// suite drives those paths, and the perft_gpu program (cli.cpp) linked
// against this library, end to end through it; it is not part of the
// product library, which has no CPU path.
#include <atomic>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/perft_b200.h"
#include "../../perft_gpu_b200/csrc/movegen.cuh"

namespace pg {
void build_tables();
int engine_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out);
}  // namespace pg

using namespace pg;

namespace {
struct VecSink {
    u32 *out;
    u32 n;
    void operator()(u32 m) { out[n++] = m; }
};

u64 perft_host(const Board &b, u32 depth)
{
    if (depth == 0) return 1;
    if (depth == 1) return count_moves<SV_KOGGE>(b);
    u32 moves[256];
    VecSink s{moves, 0};
    gen_moves<SV_KOGGE>(b, s);
    u64 total = 0;
    for (u32 i = 0; i < s.n; i++) total += perft_host(make_child(b, moves[i]), depth - 1);
    return total;
}

std::atomic<u64> g_batches{0}, g_positions{0};
std::atomic<long long> g_fail_after{-1};  // batches left before an injected failure; -1 never
std::atomic<int> g_fail_status{PERFT_ERR_CUDA};
std::atomic<u64> g_scale{1};  // every count is multiplied by this (totals beyond 64 bits on small trees)
}  // namespace

int pg::engine_batch_host(const u64 *pos, const uint8_t *depths, u32 n, u64 *out)
{
    if (n == 0) return PERFT_OK;
    long long left = g_fail_after.load();
    if (left == 0) return g_fail_status.load();
    if (left > 0) g_fail_after.store(left - 1);
    for (u32 i = 0; i < n; i++) {
        if (depths[i] > 20) return PERFT_ERR_INVALID_ARG;
        out[i] = perft_host(from_pos48(pos + 6ull * i), depths[i]) * g_scale.load();
    }
    g_batches += 1;
    g_positions += n;
    return PERFT_OK;
}

extern "C" {

int hostapi_init(void)
{
    build_tables();
    return 0;
}

// Batches and positions the stand-in engine has counted since the last reset.
void hostapi_counters(uint64_t *batches, uint64_t *positions)
{
    *batches = g_batches.load();
    *positions = g_positions.load();
}

void hostapi_reset_counters(void)
{
    g_batches = 0;
    g_positions = 0;
}

// The engine call after `batches` more successful ones returns `status`
// (a host-side failure: nothing runs on a device); -1 switches it off.
void hostapi_fail_after(long long batches, int status)
{
    g_fail_status = status;
    g_fail_after = batches;
}

// Multiplies every count by `factor` (1 restores true counts): a small tree
// then stands for one whose totals need more than 64 bits.
void hostapi_scale(uint64_t factor)
{
    g_scale = factor;
}

const char *perft_status_string(int status)
{
    return status == PERFT_OK ? "ok" : "error (host test build)";
}

// Engine lifecycle and the single-position call, for the command-line
// program built against this library.  HOSTAPI_FAIL_DEVICE=<d> makes every
// engine batch of a process initialised on device d fail with
// PERFT_ERR_CUDA (the shard processes of a split run get device = shard);
// HOSTAPI_SCALE=<k> multiplies every count by k.
void perft_config_default(perft_config *cfg)
{
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->sliders_expand = PERFT_SLIDERS_AUTO;
    cfg->sliders_leaf = PERFT_SLIDERS_AUTO;
}

int perft_init(const perft_config *cfg)
{
    build_tables();
    const char *fail = getenv("HOSTAPI_FAIL_DEVICE");
    if (fail && cfg && cfg->device == atoi(fail)) hostapi_fail_after(0, PERFT_ERR_CUDA);
    if (const char *k = getenv("HOSTAPI_SCALE")) hostapi_scale(strtoull(k, nullptr, 10));
    return PERFT_OK;
}

int perft_shutdown(void)
{
    return PERFT_OK;
}

int perft(const perft_pos48 *pos, uint32_t depth, uint64_t *out)
{
    if (!pos || !out || depth > 20) return PERFT_ERR_INVALID_ARG;
    const uint8_t d = (uint8_t)depth;
    return engine_batch_host(pos->bb, &d, 1, out);
}
}
