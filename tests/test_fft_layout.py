"""Host-side checks of the FFT core's compile-time layouts (no GPU): every
mesh line length the library builds factors into its radices; the per-stage
twiddle rows and transposed runs lie inside the table, start on even entries
(16-byte aligned) and do not overlap; and a twiddle pack (the stage blocks
one transform reads, packed for shared memory) holds each of its stages'
blocks at an even position, back to back, with the table's offsets.  The
checks run in a host program compiled by nvcc against csrc/fft_core.cuh."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "cola_halo_b200", "csrc")

PROGRAM = r'''
#include "fft_core.cuh"
#include <cstdio>
using namespace cgfft;
static int fails = 0;
#define CHECK(c, ...) do { if (!(c)) { fails++; std::printf("FAIL " __VA_ARGS__); std::printf("\n"); } } while (0)

static void check_length(int L) {
  for (int rm : {16, 8}) {
    if (!supported_length(L, rm)) continue;
    int prod = 1;
    for (int s = 0; s < num_stages(L, rm); s++) prod *= radix_at(L, s, rm);
    CHECK(prod == L, "L=%d rm=%d radices multiply to %d", L, rm, prod);
    for (int s = 1; s < num_stages(L, rm); s++) {
      const int ns = ns_before(L, s, rm), r = radix_at(L, s, rm);
      const int off = stage_tw_offset(L, ns, r), offt = stage_twt_offset(L, ns, r);
      CHECK(off >= L && off + ns * stage_rp(r) <= stage_tw_offset(L, 0, 0),
            "L=%d rm=%d stage %d rows [%d, +%d) outside the row blocks", L, rm, s, off, ns * stage_rp(r));
      CHECK(offt >= stage_tw_offset(L, 0, 0) && offt + ns * (r - 1) <= twiddle_table_len(L),
            "L=%d rm=%d stage %d runs [%d, +%d) outside the run blocks", L, rm, s, offt, ns * (r - 1));
      CHECK(off % 2 == 0 && offt % 2 == 0, "L=%d rm=%d stage %d odd block start", L, rm, s);
    }
  }
}

template <int L, int RM, bool LM, bool LML> static void check_pack() {
  using P = TwPack<L, RM, LM, LML>;
  int pos = 0;
  for (int s = 1; s < num_stages(L, RM); s++) {
    const int ns = ns_before(L, s, RM), r = radix_at(L, s, RM);
    const bool line = s == num_stages(L, RM) - 1 ? LML : LM;
    const int b = line ? stage_twt_offset(L, ns, r) : stage_tw_offset(L, ns, r);
    const int len = line ? ns * (r - 1) : ns * stage_rp(r);
    CHECK(tw_block(L, RM, LM, LML, s, false) == b, "pack L=%d stage %d block start", L, s);
    CHECK(tw_block(L, RM, LM, LML, s, true) >= len && tw_block(L, RM, LM, LML, s, true) % 2 == 0,
          "pack L=%d stage %d block length", L, s);
    CHECK(tw_pack_pos(L, RM, LM, LML, b) == pos && pos % 2 == 0, "pack L=%d stage %d position", L, s);
    pos += tw_block(L, RM, LM, LML, s, true);
  }
  CHECK(P::entries == pos && P::bytes == 8 * pos, "pack L=%d size", L);
}

int main() {
  for (int L : {16, 24, 32, 48, 64, 72, 96, 128, 144, 192, 256, 288, 384, 512, 768, 1024})
    check_length(L);
  check_pack<768, 16, false, false>();   // x pass, 16 columns
  check_pack<768, 8, false, false>();    // x pass, 8 columns
  check_pack<384, 16, false, false>();
  check_pack<512, 16, false, true>();    // z c2r at 1024^3
  check_pack<384, 16, false, true>();    // z c2r at 768^3
  check_pack<384, 16, true, true>();     // a line-major transform
  check_pack<1024, 8, false, false>();
  std::printf(fails ? "FAILED %d\n" : "OK\n", fails);
  return fails ? 1 : 0;
}
'''


def test_fft_layouts(tmp_path):
    nvcc = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    src = tmp_path / "layout.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "layout"
    r = subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                        "arch=compute_100a,code=sm_100a", "-I", CSRC, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout[-2000:]
