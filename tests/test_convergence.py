"""Optimize::isConvergence (src/optimization/opt_base.hpp:28-43) in the Python
and C++ mirrors against the oracle's restatement, on objective sequences that
cross the 1e-5 / minstep 50 criterion of the sample drivers
(opt_macro_oc.cpp:137), including a zero objective (division by zero: never
converged) and negative objectives."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def sequences():
    rng = np.random.default_rng(3)
    # compliance settling geometrically: relative changes fall through 1e-5
    a = 10.0 + 5.0 * 0.8 ** np.arange(120)
    # noisy plateau with relative changes around the threshold
    b = 3.0 * (1.0 + 1e-5 * rng.standard_normal(120))
    c = np.concatenate([np.linspace(5, 1, 60), np.zeros(3), np.full(60, 1.0)])
    d = -a
    return [a, b, c, d]


def run_oracle(oracle, seq, eps, minstep):
    C = oracle.Convergence()
    return [C.is_convergence(f, k + 1, eps, minstep) for k, f in enumerate(seq)]


@pytest.mark.parametrize("i", range(4))
@pytest.mark.parametrize("eps,minstep", [(1e-5, 50), (1e-3, 10), (0.5, 0)])
def test_python_mirror_matches_oracle(oracle, i, eps, minstep):
    from icarat2_b200 import Optimize
    seq = sequences()[i]
    O = Optimize(4, 1, 1e-4, 1.0)
    got = []
    for k, f in enumerate(seq):
        O.optstep = k + 1
        O.object_f = f
        got.append(O.isConvergence(eps, minstep))
    assert got == run_oracle(oracle, seq, eps, minstep)


def test_cpp_mirror_matches_oracle(oracle, tmp_path):
    """header-only Optimize of include/icarat_b200.hpp (no library call)"""
    src = tmp_path / "conv.cpp"
    src.write_text(r'''
#include <cstdio>
#include "icarat_b200.hpp"
int main() {
  double eps, minstep; int n;
  if(std::scanf("%lf %lf %d", &eps, &minstep, &n) != 3) return 1;
  icarat::b200::Optimize o(4, 1, 1e-4, 1.0);
  for(int k = 0; k < n; k++) {
    double f; if(std::scanf("%lf", &f) != 1) return 1;
    o.optstep = k + 1; o.object_f = f;
    std::printf("%d\n", o.isConvergence(eps, minstep));
  }
  return 0;
}
''')
    exe = tmp_path / "conv"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           str(src), "-o", str(exe)])
    for seq in sequences():
        for eps, minstep in [(1e-5, 50), (1e-3, 10)]:
            inp = "%r %r %d\n" % (eps, minstep, len(seq)) + "\n".join(repr(float(v)) for v in seq)
            out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True,
                                 check=True).stdout.split()
            assert [int(v) for v in out] == run_oracle(oracle, seq, eps, minstep)
