// Test infrastructure: a counting 64-bit integer type.  Compiling
// perft_oracle.c as C++ with -DORACLE_OPCOUNT replaces its U64 with this
// type, so every 64-bit operation the restated reference algorithm executes
// (and, or, xor, not, shifts, add, sub, mul, compares/tests, popcount, bit
// scan) increments g_ops.  Constants and loads are free.
#pragma once
#include <cstdint>

extern uint64_t g_ops;

struct U64 {
    uint64_t v;
    U64() : v(0) {}
    U64(unsigned long x) : v(x) {}
    U64(unsigned long long x) : v(x) {}
    U64(unsigned x) : v(x) {}
    U64(long x) : v((uint64_t)x) {}
    U64(int x) : v((uint64_t)(int64_t)x) {}
    explicit operator bool() const { g_ops++; return v != 0; }
};

#define OPC_BIN(op)                                                        \
    inline U64 operator op(U64 a, U64 b) { g_ops++; return U64(a.v op b.v); } \
    inline U64 &operator op##=(U64 &a, U64 b) { g_ops++; a.v = a.v op b.v; return a; }
OPC_BIN(&)
OPC_BIN(|)
OPC_BIN(^)
OPC_BIN(+)
OPC_BIN(-)
OPC_BIN(*)
#undef OPC_BIN

inline U64 operator<<(U64 a, int s) { g_ops++; return U64(a.v << s); }
inline U64 operator>>(U64 a, int s) { g_ops++; return U64(a.v >> s); }
inline U64 operator~(U64 a) { g_ops++; return U64(~a.v); }
inline bool operator==(U64 a, U64 b) { g_ops++; return a.v == b.v; }
inline bool operator!=(U64 a, U64 b) { g_ops++; return a.v != b.v; }
inline int popc(U64 x) { g_ops++; return __builtin_popcountll(x.v); }
inline int ctz(U64 x) { g_ops++; return __builtin_ctzll(x.v); }
inline uint64_t RAW(U64 x) { return x.v; }
#define OPS(n) (g_ops += (n))
