// elp_bond_writer.h -- writes one chain's bond bytes (host and device).
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "elp_internal.h"

namespace elp {

// Writes one chain's bond bytes [lo, hi) of a byte array in increasing order:
// eight bytes per store where the aligned 8-byte word lies inside [lo, hi),
// byte by byte in the words at either end, which the neighbouring chains
// (other threads) share.  Bytes skipped between two puts are zero.
struct BondWriter {
    uint8_t* base;
    size_t lo, hi;   // the chain's bytes
    size_t w;        // current word (byte offset, multiple of 8)
    uint64_t acc;    // its bytes so far
    ELP_HD void init(uint8_t* b, size_t l, size_t h)
    {
        base = b; lo = l; hi = h; w = l & ~(size_t)7; acc = 0;
    }
    ELP_HD void flush()
    {
        if (w >= lo && w + 8 <= hi) {
#ifdef __CUDA_ARCH__
            *reinterpret_cast<uint64_t*>(base + w) = acc;   // base is 8-byte aligned
#else
            memcpy(base + w, &acc, 8);
#endif
        } else {
            for (int k = 0; k < 8; k++)
                if (w + k >= lo && w + k < hi) base[w + k] = (uint8_t)(acc >> (8 * k));
        }
    }
    // byte v at offset g: lo <= g < hi, and g above every earlier put
    ELP_HD void put(size_t g, uint8_t v)
    {
        const size_t gw = g & ~(size_t)7;
        while (w < gw) { flush(); w += 8; acc = 0; }
        acc |= (uint64_t)v << (8 * (g & 7));
    }
    // the current word and zero words up to hi
    ELP_HD void finish()
    {
        for (;;) {
            flush();
            w += 8; acc = 0;
            if (w >= hi) break;
        }
    }
};

}  // namespace elp
