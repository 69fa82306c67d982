"""The VC-1 code lengths behind the transform RD's bit estimates
(libvc1_b200/csrc/vc1cu_entropy_lengths.h, generated from the reference's tables) against the
reference build: every direct AC code length (find_ac_vlc, encoder_entropy.cpp:182-192) of the
eight coding sets, and the escape-mode rate rule the trellis uses (trellis_rate_bits_for_set,
encoder_transform.cpp:1811-1841) restated here over those lengths, at both Escape-3 level widths."""
import os
import re

import numpy as np
import pytest

from libvc1_b200.abi import make_params
from oracle.bindings import Reference, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "libvc1_b200", "csrc",
                      "vc1cu_entropy_lengths.h")


def _tables():
    text = open(HEADER).read()
    body = re.search(r"kAcEntry\[kAcEntries\]\[5\] = \{(.*?)\};", text, re.S).group(1)
    rows = np.array([list(map(int, r)) for r in re.findall(r"\{(\d+), (\d+), (\d+), (\d+), (\d+)\}", body)])
    esc = list(map(int, re.search(r"kAcEscapeBits\[8\] = \{([^}]*)\}", text).group(1).split(",")))
    bits = np.zeros((8, 2, 64, 64), np.int32)
    max_level = np.zeros((8, 2, 64), np.int32)
    max_run = np.full((8, 2, 64), -1, np.int32)
    for s, run, level, last, b in rows:
        bits[s, last, run, level] = b
        max_level[s, last, run] = max(max_level[s, last, run], level)
        max_run[s, last, level] = max(max_run[s, last, level], run)
    return bits, max_level, max_run, esc


def test_direct_code_lengths_match_reference():
    bits, _, _, _ = _tables()
    r = Reference(make_params(64, 64))
    for s in range(8):
        for last in (0, 1):
            for run in range(64):
                for level in range(64):
                    assert bits[s, last, run, level] == r.ac_direct_bits(s, run, level, last), (s, last, run, level)


@pytest.mark.parametrize("pq", [4, 12])
def test_escape_rate_rule_matches_reference(pq):
    bits, max_level, max_run, esc = _tables()
    r = Reference(make_params(64, 64, pqindex=pq))
    level_bits = 11 if pq < 8 else 8
    max_q = (1 << level_bits) - 1

    def rate(s, run, level, last):
        mag = abs(level)
        if run < 0 or run > 63 or level == 0 or mag > max_q:
            return 1000000
        if mag < 64 and bits[s, last, run, mag]:
            return int(bits[s, last, run, mag]) + 1
        best = 1000000
        ld = int(max_level[s, last, run])
        if s != 3 and ld > 0 and mag > ld and mag - ld < 64 and bits[s, last, run, mag - ld]:
            best = esc[s] + 1 + int(bits[s, last, run, mag - ld]) + 1
        rd = int(max_run[s, last, mag]) if mag < 64 else -1
        if rd >= 0 and run > rd and bits[s, last, run - rd - 1, mag]:
            best = min(best, esc[s] + 2 + int(bits[s, last, run - rd - 1, mag]) + 1)
        return min(best, esc[s] + 2 + 1 + 6 + 1 + level_bits)

    rng = np.random.default_rng(pq)
    cases = [(s, run, lv, last) for s in range(8) for last in (0, 1) for run in (0, 1, 2, 5, 9, 14, 26, 40, 63)
             for lv in (1, 2, 3, 4, 5, 7, 9, 12, 19, 30, 47, 63, 64, 100, 255, 256, 2047)]
    cases += [(int(rng.integers(8)), int(rng.integers(64)), int(rng.integers(1, 300)), int(rng.integers(2)))
              for _ in range(2000)]
    for s, run, lv, last in cases:
        for sign in (1, -1):
            assert rate(s, run, sign * lv, last) == r.ac_rate_bits(s, run, sign * lv, last), (s, run, sign * lv, last)
