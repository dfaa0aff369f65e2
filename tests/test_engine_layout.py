"""Host-side checks of the transform engine's compile-time layout logic
(fherma-polymult_b200/csrc/ntt_engine.cuh), built with nvcc as a host program:

* every round map of every pass the library instantiates is free of shared
  memory bank conflicts (the kernels also static_assert this);
* the round-major row-table layout (row_table_pos) is a bijection within each
  level, and the position the kernels read for entry (y << t) + i, i even, is
  row_table_pos of that entry, with entry i + 1 next to it;
* the register bits per round are 4 exactly where that saves a round.

No GPU is needed; the test is skipped where nvcc is absent.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fherma-polymult_b200", "csrc")

PROGRAM = r"""
#include "ntt_engine.cuh"
#include <cstdio>
#include <vector>
using namespace fpm;

static int bad = 0;
#define CHECK(c, ...) do { if (!(c)) { ++bad; std::printf(__VA_ARGS__); std::printf("\n"); } } while (0)

template <int NSUB, int XS, class SWZ, int RB>
void rounds(const char* what) {
    CHECK((Rounds<NSUB, XS, SWZ, RB>::all_conflict_free()), "%s NSUB %d XS %d RB %d: bank conflicts", what, NSUB, XS, RB);
}

template <int NSUB>
void one() {
    // column pass: XS = 11 - NSUB, swizzle by register count; row pass: XS = 0
    constexpr int cr = col_pass_rb(NSUB), rr = row_pass_rb(NSUB);
    if constexpr (cr == 3) rounds<NSUB, 11 - NSUB, SwzCol, 3>("column");
    else rounds<NSUB, 11 - NSUB, SwzRow, 4>("column");
    rounds<NSUB, 0, SwzRow, rr>("row");
    CHECK(((NSUB + 3) / 4 < (NSUB + 2) / 3) == (cr == 4), "NSUB %d: column register bits %d", NSUB, cr);
    CHECK(rr == cr, "NSUB %d: row register bits %d", NSUB, rr);
}

int main() {
    one<6>(); one<7>(); one<8>(); one<9>(); one<10>(); one<11>();
    for (int nsub = 6; nsub <= 11; ++nsub) {
        for (int rb = 3; rb <= 4; ++rb) {
            const uint32_t S = 1u << nsub;
            std::vector<int> hit(S, 0);
            for (uint32_t e = 1; e < S; ++e) {
                const uint32_t p = row_table_pos(nsub, rb, e);
                const int le = 31 - __builtin_clz(e);
                CHECK(p < S && p >= (1u << le) && p < (2u << le), "nsub %d rb %d: entry %u leaves its level", nsub, rb, e);
                if (p < S) hit[p]++;
            }
            for (uint32_t p = 1; p < S; ++p) CHECK(hit[p] == 1, "nsub %d rb %d: position %u hit %d times", nsub, rb, p, hit[p]);
            const int count = (nsub + rb - 1) / rb;
            for (int r = 0; r < count; ++r) {
                const int cnt = (r < count - 1 || nsub % rb == 0) ? rb : nsub % rb;
                const int lo = nsub - rb * r - cnt, LY = nsub - rb - lo;
                for (int t = rb - cnt; t < rb; ++t) {
                    CHECK(table_ly(nsub, rb, LY + t) == LY, "nsub %d rb %d: level %d in round %d", nsub, rb, LY + t, r);
                    for (uint32_t y = 1u << LY; y < (2u << LY); ++y)
                        for (uint32_t m = 0; m < (1u << t); m += (t ? 2 : 1)) {
                            const uint32_t at = t >= 2 ? (1u << (LY + t)) + (m << LY) + 2u * (y - (1u << LY)) : (y << t) + m;
                            CHECK(row_table_pos(nsub, rb, (y << t) + m) == at, "nsub %d rb %d: read of (%u, %u)", nsub, rb, y, m);
                            if (t) CHECK(row_table_pos(nsub, rb, (y << t) + m + 1) == at + 1, "nsub %d rb %d: pair (%u, %u)", nsub, rb, y, m);
                        }
                }
            }
        }
    }
    std::printf("%d failures\n", bad);
    return bad != 0;
}
"""


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


def test_engine_layout(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    src = tmp_path / "layout.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "layout"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", "-I", CSRC,
                    str(src), "-o", str(exe)], check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "0 failures" in out.stdout
