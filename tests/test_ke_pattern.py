"""The coefficient pattern of the FP64 streaming K(E)u (csrc/ke_pattern.inc) is current.

ke_pattern.inc is generated from the library's own hex8 stiffness (csrc/hex8.hpp, fea.cpp:117-179) by
csrc/gen_ke_pattern.cpp.  This test rebuilds the generator with g++, checks its output against the
committed file, and checks the pattern's meaning on the oracle's Ke (the same element stiffness,
restated in C): every entry is +-(one of KE_ND magnitudes), and each column's row order is a
permutation sorted by magnitude index.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "algorithmengineering_altproject_b200", "csrc")


def parse(text, name):
    m = re.search(r"constexpr int %s\(int i\) \{\s*constexpr [a-z ]+ t\[\d+\] = \{([^}]*)\}" % name, text)
    return [int(v) for v in m.group(1).split(",")]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_committed_pattern_matches_generator(tmp_path):
    exe = str(tmp_path / "gen_ke_pattern")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(CSRC, "gen_ke_pattern.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(CSRC, "ke_pattern.inc")) as f:
        assert f.read() == out


def test_pattern_describes_the_element_stiffness():
    from oracle.bindings import Oracle
    K = np.array(Oracle(6, 12, 6, red_mode=1).ke()).reshape(-1)
    with open(os.path.join(CSRC, "ke_pattern.inc")) as f:
        text = f.read()
    nd = int(re.search(r"KE_ND = (\d+);", text).group(1))
    idx, neg, first, order = (parse(text, n) for n in ("ke_idx", "ke_neg", "ke_first", "ke_row_order"))
    D = np.abs(K[first])
    assert len(D) == nd == len(set(D.tolist()))
    rebuilt = np.where(np.array(neg) == 1, -D[idx], D[idx])
    assert np.array_equal(rebuilt.view(np.int64), K.view(np.int64))
    for j in range(24):
        rows = order[24 * j:24 * j + 24]
        assert sorted(rows) == list(range(24))
        keys = [idx[24 * q + j] for q in rows]
        assert keys == sorted(keys)
