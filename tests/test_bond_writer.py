"""The chain walk's bond writer (csrc/elp_bond_writer.h), compiled for the
host: eight-byte stores inside a chain's bytes, single bytes in the words it
shares with its neighbours, zeros between puts.  Checked against plain
byte-by-byte writes over many chain lengths, chain counts and early stops,
under the address and undefined-behaviour sanitizers (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "mc-polymer-simulation_b200", "csrc")

DRIVER = r"""
#include <stdio.h>
#include <string.h>
#include <vector>
#include "elp_bond_writer.h"

static uint64_t s = 88172645463325252ull;
static uint64_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }

int main() {
    long cases = 0;
    for (int N = 1; N <= 70; N++)
        for (int P = 1; P <= 9; P++)
            for (int rep = 0; rep < 30; rep++) {
                std::vector<uint8_t> ref((size_t)P * N + 16, 0xAB), got((size_t)P * N + 16, 0xAB);
                for (int p = 0; p < P; p++) {
                    elp::BondWriter bw;
                    bw.init(got.data(), (size_t)p * N, (size_t)p * N + N);
                    const long lim = N - (long)(rnd() % (unsigned)N);   // the zeros of the head run's offset
                    const bool early = rnd() % 5 == 0;                  // a walk that stops on a bad chain
                    for (int k = 0; k < N; k++) ref[(size_t)p * N + k] = 0;
                    long i = 0;
                    while (i < lim) {
                        long here = 1 + (long)(rnd() % 4 == 0 ? rnd() % 20 : rnd() % 2);
                        if (i + here > lim) here = lim - i;
                        const uint8_t v = (uint8_t)(1 + rnd() % 14);
                        bw.put((size_t)p * N + (size_t)(i + here - 1), v);
                        ref[(size_t)p * N + (size_t)(i + here - 1)] = v;
                        i += here;
                        if (early && rnd() % 7 == 0) break;
                    }
                    bw.finish();
                }
                if (memcmp(ref.data(), got.data(), ref.size()) != 0) {
                    printf("mismatch N=%d P=%d\n", N, P);
                    return 1;
                }
                cases++;
            }
    printf("ok %ld\n", cases);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_bond_writer_matches_byte_writes(tmp_path):
    src = tmp_path / "bw.cpp"
    exe = tmp_path / "bw"
    src.write_text(DRIVER)
    flags = ["-O1", "-fsanitize=address,undefined", "-fno-sanitize-recover=all"]
    subprocess.run(["g++", *flags, "-I", CSRC, str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok 18900"), out.stdout
