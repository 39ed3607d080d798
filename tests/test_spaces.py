"""The k segmentation of the update kernels' thread spaces
(courant_b200/csrc/spaces.hpp): thin segments join a neighbour without
turning a thick CPML-free segment into a CPML one."""
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    exe = tmp_path_factory.mktemp("spaces") / "spaces_case"
    subprocess.run(["g++", "-std=c++17", "-O1", str(ROOT / "tests" / "spaces_case.cpp"), "-o", str(exe)], check=True)

    def run(end, slab, box, cuts):
        out = subprocess.run([str(exe), str(end), *map(str, slab), *map(str, box), *map(str, cuts)],
                             capture_output=True, text=True, check=True).stdout
        return [int(v) for v in out.split()]
    return run


def test_large_board_h_column(case):
    # H of the 1500 x 1014 x 64 board: z CPML cells 56-63, k groups to 68
    assert case(68, (56, 64), (0, 0), [56, 64]) == [0, 56, 68]


def test_large_board_e_column(case):
    # E: Debye boxes end at 48, z CPML nodes 56-64 (cut at 68 = end)
    assert case(68, (56, 65), (0, 48), [48, 56]) == [0, 56, 68]


def test_thin_plain_joins_box_not_slab(case):
    assert case(100, (80, 100), (0, 40), [40, 48, 80]) == [0, 48, 80, 100]


def test_thick_segments_stay(case):
    assert case(88, (72, 88), (0, 24), [24, 72]) == [0, 24, 72, 88]


def test_no_cuts_and_single_segment(case):
    assert case(68, (0, 0), (0, 0), []) == [0, 68]
    assert case(12, (0, 0), (0, 0), []) == [0, 12]


def test_thin_box_does_not_turn_a_thick_plain_segment_into_debye(case):
    # E of the lossy 2-port line: Debye boxes k 0-11 under 64 plain node groups, z CPML from 76
    assert case(88, (76, 87), (0, 12), [12, 76]) == [0, 12, 76, 88]


def test_z_tails_keep_a_thin_box_out_of_the_slab_segment(case):
    # E of the lossy 2-port line with z tails (no cut at the slab): the thin Debye box stays
    # apart instead of moving the thick air-and-slab segment into the Debye kernel
    assert case(-88, (76, 87), (0, 12), [12]) == [0, 12, 88]
    # a thin air segment between a thick box and the slab-and-air top joins the box (the Debye
    # kernel takes points outside the box), never making the top general
    assert case(-88, (76, 87), (0, 40), [40, 48]) == [0, 48, 88]
    # a thin slab-and-air top above a thick box joins it (the Debye kernel takes the tail's groups)
    assert case(-88, (76, 87), (0, 76), [76]) == [0, 88]


def test_z_tails_large_board_columns(case):
    assert case(-68, (56, 64), (0, 0), []) == [0, 68]
    assert case(-68, (56, 65), (0, 48), [48]) == [0, 48, 68]
