"""The fused RBL kernel's shortcuts of the batch test, compiled for the host
from the same header the kernels use (rbmd_b200/csrc/rbx_common.cuh).

RblShellSampleSelected keeps a shell pair when MixRblSampleKey(key) % freq
== 0 (rbl_full_neighbor_list_op.hip.cu:6-30).  The kernels never form that
modulus: for freq <= 4 they read two bits of a partial hash, for other freq
they use a divisibility test by multiplication.  Both are checked here
against the full 64-bit mix and the % operator on 2^21 random keys (plus
edge keys) for every freq from 1 to 40.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "rbmd_b200", "csrc")

PROG = r"""
#include <cstdio>
#include <cstdlib>
#include "rbx_common.cuh"
using namespace rbx;
int main(int argc, char** argv) {
  FILE* f = fopen(argv[1], "rb");
  long n = atol(argv[2]);
  unsigned long long* k = (unsigned long long*)malloc(8 * n);
  if (fread(k, 8, n, f) != (size_t)n) return 2;
  fclose(f);
  long bad = 0;
  for (int freq = 1; freq <= 40; ++freq) {
    const DivTest t = make_divtest(freq);
    const bool pow2 = (freq & (freq - 1)) == 0;
    for (long i = 0; i < n; ++i) {
      const unsigned long long h = rbl_mix(k[i]);
      const bool want = h % (unsigned long long)freq == 0;
      if (divisible(h, t) != want) ++bad;
      if (pow2 && freq <= 4 && rbl_selected_low2(k[i], (unsigned)(freq - 1)) != want) ++bad;
    }
  }
  printf("%ld\n", bad);
  return 0;
}
"""


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


@pytest.mark.skipif(_nvcc() is None, reason="nvcc not available")
def test_batch_test_shortcuts_match_full_hash(tmp_path):
    src = tmp_path / "hash.cu"
    src.write_text(PROG)
    exe = tmp_path / "hash"
    subprocess.run([_nvcc(), "-O2", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe)], check=True, capture_output=True)
    rng = np.random.default_rng(20261203)
    keys = rng.integers(0, 2 ** 63, size=1 << 21, dtype=np.int64).astype(np.uint64)
    keys[::2] ^= np.uint64(1) << np.uint64(63)
    edge = np.array([0, 1, 2 ** 32 - 1, 2 ** 32, 2 ** 64 - 1, 0x9e3779b97f4a7c15,
                     2 ** 64 - 0x9e3779b97f4a7c15], dtype=np.uint64)
    keys[:len(edge)] = edge
    kf = tmp_path / "keys.bin"
    keys.tofile(kf)
    out = subprocess.run([str(exe), str(kf), str(len(keys))], check=True, capture_output=True,
                         text=True).stdout
    assert int(out.strip()) == 0
