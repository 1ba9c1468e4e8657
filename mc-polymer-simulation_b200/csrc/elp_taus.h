// elp_taus.h -- the four-component Tausworthe generator (L'Ecuyer's
// LFSR113 shifts and masks) with the seeding of the reference's util/rng.h:
// the host programs that must reproduce the reference's own fixed random
// streams (scaleup's path choices, tuv2pov's light placement) draw from it.
#pragma once
#include <stdint.h>

struct elp_taus {
    uint32_t s[4];
    explicit elp_taus(uint32_t seed) : s{seed, seed ^ 0xa741f123u, seed ^ 0x213910abu, seed ^ 0xcd123e14u} {}
    uint32_t next()
    {
        uint32_t b;
        b = ((s[0] << 6) ^ s[0]) >> 13;  s[0] = ((s[0] & 0xFFFFFFFEu) << 18) ^ b;
        b = ((s[1] << 2) ^ s[1]) >> 27;  s[1] = ((s[1] & 0xFFFFFFF8u) << 2) ^ b;
        b = ((s[2] << 13) ^ s[2]) >> 21; s[2] = ((s[2] & 0xFFFFFFF0u) << 7) ^ b;
        b = ((s[3] << 3) ^ s[3]) >> 12;  s[3] = ((s[3] & 0xFFFFFF80u) << 13) ^ b;
        return s[0] ^ s[1] ^ s[2] ^ s[3];
    }
    // floor(n * u) for u = next() / 2^32, exact in double for the n used here
    int below(int n) { return (int)(((uint64_t)next() * (uint64_t)n) >> 32); }
    // u = next() / 2^32 in [0, 1), exact
    double uniform() { return (double)next() * (1.0 / 4294967296.0); }
};
