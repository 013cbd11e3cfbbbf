// MT19937 output streams for one thread (Matsumoto & Nishimura 1998), seeded with
// init_genrand(seed): mt[0] = seed, mt[i] = 1812433253*(mt[i-1] ^ mt[i-1]>>30) + i, the
// seeding recurrence the reference's twisters use (oplib/opcuda/smc.cu:127-131).
//
// Keyed seeding (key1 != 0): the same recurrence with key1 added to mt[1] before the
// recurrence continues from it (mt[1] = 1812433253*(seed ^ seed>>30) + 1 + key1).  Two
// (seed, key1) pairs give equal initial states only if both members are equal, so one
// seed yields 2^32 distinct generators; key1 = 0 is init_genrand(seed).
//
// Two forms, bit-identical on the outputs they share:
//
// mt19937_first (n <= 623): the whole generator in registers.  The first 623 outputs of
// a freshly seeded MT19937 only need one regeneration of the state, and every regenerated
// word is an XOR of tw() terms of initial words mt[j], each of which is a forward
// recurrence from the seed.  The function walks that recurrence with a few cursors (and
// one saved word, mt[397]) instead of storing 624 words, so it uses no local or shared
// memory:
//   i <  227 : mt'[i] = mt[i+397] ^ tw(mt[i], mt[i+1])
//   i <  454 : mt'[i] = mt[i+170] ^ tw(mt[i-227], mt[i-226]) ^ tw(mt[i], mt[i+1])
//   i <  623 : mt'[i] = mt[i-57] ^ tw(mt[i-454], mt[i-453]) ^ tw(mt[i-227], mt[i-226])
//                       ^ tw(mt[i], mt[i+1])
// Output 623 would need mt'[0] as the second operand of its tw(), i.e. a word of the
// regenerated state, which is where the cursor form stops.
//
// mt19937_any (any n): the first 623 outputs come from the same cursors, and each
// regenerated word is also stored in a per-thread 624-word array (local memory on the
// device, 2496 bytes a thread), so no separate initialisation pass is needed.  Output 623
// closes the first regeneration (mt'[623] = mt'[396] ^ tw(mt[623], mt'[0]), with the
// initial word mt[623] taken from the cursor), and every later output regenerates one word
// of the array:
//   mt[i] = mt[(i+397) mod 624] ^ tw(mt[i], mt[(i+1) mod 624]);  output temper(mt[i])
// Word i of a generation reads mt[i+397] before it is regenerated (i < 227) and after
// (i >= 227), and word 623 reads the regenerated mt[0], exactly as genrand_int32's block
// refill does, so the stream is MT19937's for every n.
//
// The header compiles as plain C++ too, so the host can check both forms against an
// independent MT19937.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define OPB_MT_FN __host__ __device__ __forceinline__
#else
#define OPB_MT_FN inline
#endif

namespace opb {

// Longest stream mt19937_first serves.
constexpr int kMtCursorMax = 623;

OPB_MT_FN uint32_t mt_init_next(uint32_t v, uint32_t i) {
    return 1812433253u * (v ^ (v >> 30)) + i;
}
OPB_MT_FN uint32_t mt_tw(uint32_t a, uint32_t b) {
    uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return (y >> 1) ^ ((b & 1u) ? 0x9908b0dfu : 0u);
}
OPB_MT_FN uint32_t mt_temper(uint32_t y) {
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

// Calls f(k, w_k) with the regenerated (untempered) state word w_k = mt'[k] for the first
// n (<= 623) words of MT19937 seeded with (seed, key1); returns the initial word mt[n].
template <class F>
OPB_MT_FN uint32_t mt19937_cursor_words(uint32_t seed, uint32_t key1, int n, F &&f) {
    const uint32_t m1 = mt_init_next(seed, 1u) + key1;
    // cursor A at i: (a0, a1) = (mt[i], mt[i+1])
    uint32_t a0 = seed, a1 = m1;
    // cursor B at i + 397
    uint32_t b = m1;
#pragma unroll 1
    for (uint32_t j = 2; j <= 397; j++) b = mt_init_next(b, j);
    const uint32_t m397 = b;
    uint32_t bi = 397;
    int i = 0;
    const int n1 = n < 227 ? n : 227;
#pragma unroll 1
    for (; i < n1; i++) {
        f(i, b ^ mt_tw(a0, a1));
        a0 = a1; a1 = mt_init_next(a1, (uint32_t)i + 2u);
        bi++; b = mt_init_next(b, bi);
    }
    if (i >= n) return a0;
    // phase 2: cursor C at i-227 from the seed, cursor B restarted at 397
    uint32_t c0 = seed, c1 = m1;
    b = m397; bi = 397;
    const int n2 = n < 454 ? n : 454;
#pragma unroll 1
    for (; i < n2; i++) {
        f(i, b ^ mt_tw(c0, c1) ^ mt_tw(a0, a1));
        a0 = a1; a1 = mt_init_next(a1, (uint32_t)i + 2u);
        c0 = c1; c1 = mt_init_next(c1, (uint32_t)(i - 227) + 2u);
        bi++; b = mt_init_next(b, bi);
    }
    if (i >= n) return a0;
    // phase 3: cursor D at i-454 from the seed, B restarted at 397 (= i-57 at i = 454)
    uint32_t d0 = seed, d1 = m1;
    b = m397; bi = 397;
#pragma unroll 1
    for (; i < n; i++) {
        f(i, b ^ mt_tw(d0, d1) ^ mt_tw(c0, c1) ^ mt_tw(a0, a1));
        a0 = a1; a1 = mt_init_next(a1, (uint32_t)i + 2u);
        c0 = c1; c1 = mt_init_next(c1, (uint32_t)(i - 227) + 2u);
        d0 = d1; d1 = mt_init_next(d1, (uint32_t)(i - 454) + 2u);
        bi++; b = mt_init_next(b, bi);
    }
    return a0;
}

// Calls f(k, x_k) for the first n (<= 623) outputs of MT19937 seeded with (seed, key1).
template <class F>
OPB_MT_FN void mt19937_first(uint32_t seed, uint32_t key1, int n, F &&f) {
    mt19937_cursor_words(seed, key1, n, [&](int i, uint32_t w) { f(i, mt_temper(w)); });
}

// Calls f(k, x_k) for the first n outputs of MT19937 seeded with (seed, key1), any n >= 0.
template <class F>
OPB_MT_FN void mt19937_any(uint32_t seed, uint32_t key1, int n, F &&f) {
    uint32_t mt[624];
    const int n1 = n < kMtCursorMax ? n : kMtCursorMax;
    const uint32_t init623 = mt19937_cursor_words(seed, key1, n1, [&](int k, uint32_t w) {
        mt[k] = w;
        f(k, mt_temper(w));
    });
    if (n <= kMtCursorMax) return;
    mt[623] = mt[396] ^ mt_tw(init623, mt[0]);
    f(623, mt_temper(mt[623]));
    int i = 0, im = 397;  // im = (i + 397) mod 624
    uint32_t cur = mt[0]; // mt[i], carried from the previous output's mt[i+1] load
#pragma unroll 1
    for (int k = 624; k < n; k++) {
        const int i1 = i == 623 ? 0 : i + 1;
        const uint32_t nxt = mt[i1];
        const uint32_t y = mt[im] ^ mt_tw(cur, nxt);
        mt[i] = y;
        f(k, mt_temper(y));
        i = i1;
        im = im == 623 ? 0 : im + 1;
        cur = nxt;
    }
}

// mt19937_first when ANY_LENGTH is false (n <= 623), mt19937_any otherwise.
template <bool ANY_LENGTH, class F>
OPB_MT_FN void mt19937_stream(uint32_t seed, uint32_t key1, int n, F &&f) {
    if constexpr (ANY_LENGTH) mt19937_any(seed, key1, n, static_cast<F &&>(f));
    else mt19937_first(seed, key1, n, static_cast<F &&>(f));
}

}  // namespace opb
