"""The two-phase correctly rounded log and cos of the Gaussian draws
(gauge_higgs_b200/csrc/gh_rng.cuh, compiled for the host): the first phase returns a
value only when its error bound settles the rounding, so it must equal the
double-double evaluation on every argument.  Checked on 2 million arguments of the
draws' own distribution (u1, 2 pi u2 from the counter RNG) and on arguments next to the
hard spots (u near 1 and near 1/sqrt 2; x near the multiples of pi/2, where cos x is
small).  The GPU kernels compile the same functions."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r'''
#include "gh_rng.cuh"
#include <cstdio>
using namespace ghrng;
int main() {
  long bad_log = 0, bad_cos = 0, n = 0;
  for (long i = 0; i < 2000000; ++i) {
    const double u1 = uniform(77, splitmix64(2 * i + 1)), u2 = uniform(77, splitmix64(2 * i + 2));
    const double x = mul_rn(6.283185307179586, u2);
    bad_log += cr_log_fast(u1) != cr_log(u1);
    bad_cos += cr_cos_fast(x) != cr_cos(x);
    const double v = 1.0 - u2 * 1e-6, w = 0.7071067811865476 + (u2 - 0.5) * 1e-9;
    bad_log += cr_log_fast(v) != cr_log(v);
    bad_log += cr_log_fast(w) != cr_log(w);
    const double xq = 1.5707963267948966 * (1 + (int)(u1 * 3.999)) + (u2 - 0.5) * 1e-7;
    bad_cos += cr_cos_fast(xq) != cr_cos(xq);
    ++n;
  }
  std::printf("%ld %ld %ld\n", n, bad_log, bad_cos);
  return 0;
}
'''


def test_first_phase_equals_double_double(tmp_path):
    src, exe = tmp_path / "rng_twophase.cpp", tmp_path / "rng_twophase"
    src.write_text(SRC)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    "-I" + os.path.join(ROOT, "gauge_higgs_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    n, bad_log, bad_cos = map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.split())
    assert n == 2000000
    assert bad_log == 0 and bad_cos == 0, (bad_log, bad_cos)
