// Measurement infrastructure: integer-pipe peak of the current GPU.
//
// The perft kernels are bound by 32-bit integer/logic throughput (64-bit
// bitboard operations split into LOP3 / SHF / IADD3 / POPC instructions).
// This probe issues long dependent-free streams of those instructions and
// reports the achieved operations per second, the denominator of the
// integer roofline.  Built as its own library (libperft_probe.so); the
// engine does not use it.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int NT = 256;
constexpr int CHAINS = 8;

// kind 0: LOP3 (3-input logic), kind 1: integer add, kind 2: LOP3/add/SHF
// mix, kind 3: IMAD (integer multiply-add, the FMA pipe), kind 4: LOP3 and
// IMAD alternating (both integer pipes), kind 5: IMAD.HI, kind 6: IMAD.WIDE
// (plus the LOP3 that folds its two result words).  Inline PTX keeps the compiler from
// folding the chains.
template <int KIND>
__global__ void __launch_bounds__(NT) k_probe(uint32_t *out, uint32_t seed, int iters)
{
    uint32_t a[CHAINS], b = seed ^ threadIdx.x, c = seed * 2654435761u + blockIdx.x;
#pragma unroll
    for (int i = 0; i < CHAINS; i++) a[i] = seed + i * 0x9E3779B9u + threadIdx.x;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < CHAINS; i++) {
            uint32_t r = a[i];
            if (KIND == 0) {
                asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
            } else if (KIND == 1) {
                asm volatile("add.u32 %0, %1, %2;" : "=r"(r) : "r"(r), "r"(b));
            } else if (KIND == 2) {
                asm volatile("lop3.b32 %0, %1, %2, %3, 0x78;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
                asm volatile("add.u32 %0, %1, %2;" : "=r"(r) : "r"(r), "r"(c));
                asm volatile("shf.l.wrap.b32 %0, %1, %2, 7;" : "=r"(r) : "r"(r), "r"(b));
            } else if (KIND == 3) {
                asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
            } else if (KIND == 4) {
                asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
                asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
            } else if (KIND == 5) {
                asm volatile("mad.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(r), "r"(b), "r"(c));
            } else {
                uint64_t w;
                asm volatile("mad.wide.u32 %0, %1, %2, %3;" : "=l"(w) : "r"(r), "r"(b), "l"((uint64_t)c));
                r = (uint32_t)w ^ (uint32_t)(w >> 32);
            }
            a[i] = r;
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < CHAINS; i++) s ^= a[i];
    if (s == 0x12345678u) out[blockIdx.x * NT + threadIdx.x] = s;
}

template <int KIND>
double run(int device, int opsPerChainStep)
{
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return -1.0;
    int perSm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_probe<KIND>, NT, 0);
    if (perSm < 1) perSm = 1;
    const int blocks = prop.multiProcessorCount * perSm;
    uint32_t *out = nullptr;
    if (cudaMalloc(&out, sizeof(uint32_t) * blocks * NT) != cudaSuccess) return -1.0;
    const int iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_probe<KIND><<<blocks, NT>>>(out, 1u, 256);  // warm-up
    cudaEventRecord(e0);
    k_probe<KIND><<<blocks, NT>>>(out, 7u, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double ops = (double)blocks * NT * iters * CHAINS * opsPerChainStep;
    return ops / (ms * 1e-3);
}

}  // namespace

extern "C" {

// Writes the measured 32-bit integer instructions per second (per lane) for
// seven instruction mixes: LOP3, add, LOP3+add+SHF, IMAD, LOP3+IMAD,
// IMAD.HI, IMAD.WIDE+LOP3.  Returns 0 on success.
int perft_int32_peak_probe(int device, double out[7])
{
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    out[0] = run<0>(device, 1);
    out[1] = run<1>(device, 1);
    out[2] = run<2>(device, 3);
    out[3] = run<3>(device, 1);
    out[4] = run<4>(device, 2);
    out[5] = run<5>(device, 1);
    out[6] = run<6>(device, 2);
    for (int i = 0; i < 7; i++)
        if (out[i] <= 0) return -1;
    return 0;
}
}
