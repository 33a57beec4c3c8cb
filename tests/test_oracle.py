"""The oracle (C++ restatement, oracle/dr_oracle.cpp) pinned to the reference.

Each golden fixture holds the compiled reference's own forward image, backward
image and every gradient for a seeded scene (tests/golden/make_golden.py).  The
oracle, drawing random numbers exactly as the reference does, must reproduce
them to float round-off.
"""
import numpy as np
import pytest

from conftest import build_golden_scene, golden_cases, load_golden, rel_err
import oracle

TOL = 2e-5  # max |diff| / max |ref|: float round-off of a different summation order


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_fixture(case, ltc_table):
    meta, gold = load_golden(case)
    wl = build_golden_scene(meta)
    from golden.make_golden import scene_checksum
    assert scene_checksum(wl) == meta["checksum"], "scene builder changed since the fixture was made"
    fwd = oracle.oracle_render(wl, meta["seed"], rng_mode=oracle.REFERENCE, cores=meta["cores"],
                               ltc_table=ltc_table, shape_rank=gold["shape_rank"])
    assert rel_err(fwd["image"], gold["image"]) < TOL
    bwd = oracle.oracle_render(wl, meta["seed"], d_image=gold["d_image"], rng_mode=oracle.REFERENCE,
                               cores=meta["cores"], ltc_table=ltc_table, shape_rank=gold["shape_rank"])
    assert rel_err(bwd["image"], gold["image_bwd"]) < TOL
    assert rel_err(bwd["grad"], gold["grad"]) < TOL
    # the fixture exercises the backward machinery
    assert bwd["stats"][0] > 0 and bwd["stats"][1] > 0
    assert np.abs(gold["grad"]).max() > 0


def test_philox_known_answers():
    """Random123 known-answer vectors of Philox4x32-10."""
    assert [hex(x) for x in oracle.philox_raw([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox_raw([0xffffffff] * 4, [0xffffffff] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox_raw([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                              [0xa4093822, 0x299f31d0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_philox_stream_is_uniform():
    u = oracle.philox(7, 0, 12345, 0, 100000)
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.005
    assert abs(u.var() - 1.0 / 12.0) < 0.002


def test_oracle_philox_mode_is_deterministic_and_unbiased():
    """Philox streams give the same image as reference order up to noise."""
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(seed=0, resolution=(24, 24), spp=64)
    a = oracle.oracle_render(wl, 3, rng_mode=oracle.PHILOX)["image"]
    b = oracle.oracle_render(wl, 3, rng_mode=oracle.PHILOX)["image"]
    assert np.array_equal(a, b)
    c = oracle.oracle_render(wl, 3, rng_mode=oracle.REFERENCE)["image"]
    assert abs(a.mean() - c.mean()) < 0.02 * c.mean()
