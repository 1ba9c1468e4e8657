/*
 * philox_ref.c -- TEST INFRASTRUCTURE ONLY.
 * Philox4x32-10 counter-based generator, written from the round function
 * published by Salmon, Moraes, Dror and Shaw, "Parallel Random Numbers: As
 * Easy as 1, 2, 3" (SC'11): per round, two 32x32->64 products of counter
 * words with the multipliers 0xD2511F53 / 0xCD9E8D57, a word permutation
 * with key xor, and a Weyl key bump by 0x9E3779B9 / 0xBB67AE85.
 */
#include "oracle.h"

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
