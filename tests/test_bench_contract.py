"""bench.py's reporting helpers, on CPU: the roofline's `traffic` comes from
the committed ncu summaries, so every kernel key the headline line can ask
for must resolve, and every summary must carry the command that made it."""
from __future__ import annotations

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_headline_traffic_keys_resolve():
    # the A kernel of the headline system for each layout the solver can pick
    for key in ("cg_a_ell8_laplace1024", "cg_a_codec_laplace1024", "cg_a_row_laplace1024"):
        t = bench.ncu_traffic(key)
        assert t is not None and t > 1e6, key
    assert bench.ncu_traffic("no_such_kernel") is None


def test_cg_a_kernel_name_follows_the_layout():
    assert bench.cg_a_kernel_name(0, 9).startswith("cg_a_ell8_kernel")
    for rb in (33, 49, 65):
        assert bench.cg_a_kernel_name(0, rb).startswith("cg_a_ellv_kernel")
    assert bench.cg_a_kernel_name(3, 4).startswith("cg_a_codec_kernel")
    assert bench.cg_a_kernel_name(10, 4).startswith("cg_a_codec_kernel")
    assert bench.cg_a_kernel_name(12, 4).startswith("cg_a_kernel")


def test_profile_summaries_are_short_text_with_their_command():
    d = os.path.join(ROOT, "profiles")
    names = sorted(os.listdir(d))
    assert names
    for fn in names:
        assert fn.endswith((".txt", ".md")), fn
        path = os.path.join(d, fn)
        assert os.path.getsize(path) < 16 * 1024, fn
        text = open(path).read()
        assert "Command" in text, fn
        assert "--clock-control none" in text, fn
