"""bench.py's exp2/reciprocal floor of the short range (`roofline.xu`), on CPU.

The two-slot short range evaluates two sources per non-home stencil cell,
each with one exp2 and one reciprocal, for every body; the floor is that
operation count at the MUFU unit's 16 results per clock per SM. The list form
(an exact limit other than 2, or under one body per two cells) has no such
fixed count, and the floor is then absent.
"""

import sys
import types
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


@pytest.fixture
def b200_props(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "get_device_properties",
                        lambda i: types.SimpleNamespace(multi_processor_count=148))


def test_two_slot_floor_counts_four_mufu_per_cell(b200_props):
    sc = bench.make_workload("plummer_walls")  # 400k bodies on 512x256 cells: the two-slot form
    xu = bench.short_range_xu(sc, 0.05, {"sm_mhz": 1965.0})
    assert xu["ops_per_launch"] == 4 * 48 * sc.n  # 7x7 stencil less the home cell
    want_ms = 4 * 48 * sc.n / (16 * 148 * 1965e6) * 1e3
    assert xu["floor_ms"] == pytest.approx(want_ms, rel=1e-12)
    assert xu["frac"] == pytest.approx(want_ms / 0.05, rel=1e-12)


def test_list_form_and_missing_clock_have_no_floor(b200_props):
    sparse = bench.make_workload("uniform_torus")  # 50k bodies on 131k cells: the list form
    assert bench.short_range_xu(sparse, 0.02, {"sm_mhz": 1965.0}) is None
    dense = bench.make_workload("plummer_walls")
    assert bench.short_range_xu(dense, 0.05, {"sm_mhz": None, "sm_max_mhz": None}) is None
    assert bench.short_range_xu(dense, 0.0, {"sm_mhz": 1965.0}) is None
