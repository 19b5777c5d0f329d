"""The oracle and the host layer against the reference's own known-answer
tests (fixtures in tests/golden, made by tests/golden/make_golden.py)."""
from __future__ import annotations

import json
import struct
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _f32(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def test_f16_known_values_oracle_and_host(pkg, oracle):
    kat = json.loads((GOLDEN / "f16_kat.json").read_text())
    assert len(kat["exact"]) + len(kat["masked"]) == 11
    host = pkg._native.lib().oxpt_f32_to_f16
    for e in kat["exact"]:
        v = _f32(e["f32_bits"])
        assert oracle.f32_to_f16(v) == e["f16"], e
        assert host(v) == e["f16"], e
    for e in kat["masked"]:
        v = _f32(e["f32_bits"])
        assert oracle.f32_to_f16(v) & e["mask"] == e["f16"], e
        assert host(v) & e["mask"] == e["f16"], e


def test_f16_matches_numpy_round_to_nearest_even(pkg, oracle):
    """Beyond the KAT: every finite value rounds like IEEE binary16 RNE."""
    rng = np.random.default_rng(3)
    vals = np.concatenate([rng.standard_normal(4000) * 1e3, rng.uniform(-1e-4, 1e-4, 4000),
                           rng.uniform(-7e4, 7e4, 2000)]).astype(np.float32)
    host = pkg._native.lib().oxpt_f32_to_f16
    want = vals.astype(np.float16).view(np.uint16)
    got = np.array([host(float(v)) for v in vals], np.uint16)
    assert np.array_equal(got, want)
    got_o = np.array([oracle.f32_to_f16(float(v)) for v in vals[:2000]], np.uint16)
    assert np.array_equal(got_o, want[:2000])


@pytest.mark.parametrize("strategy", [0, 1, 2])
def test_white_furnace_oracle(pkg, oracle, strategy):
    """tests/pathtrace.rs white_furnace: L = Le / (1 - rho) = 2.0 +- 0.04 for
    MIS, light-only and BSDF-only, through the oracle."""
    g = json.loads((GOLDEN / "furnace.json").read_text())
    opts = pkg.RenderOptions(width=g["width"], height=g["height"], ambient=g["ambient"],
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=g["spp"], max_bounces=g["bounces"],
                                                             strategy=strategy))
    p = pkg.prepare(pkg.Scene.furnace(g["rho"], g["le"]), opts)
    cam = g["camera"]
    # The furnace scene's camera is the reference test's.
    assert np.allclose(np.array(p.params.eye[:3]), cam["eye"], atol=1e-6)
    acc, _ = oracle.render(p, g["spp"])
    assert np.all(acc[..., 3] == g["spp"])
    mean = (acc[..., :3] / acc[..., 3:4]).mean(axis=(0, 1))
    assert np.all(np.abs(mean - g["expected"]) < g["tolerance"]), mean


def test_constants_match_reference(pkg):
    c = json.loads((GOLDEN / "pt_constants.json").read_text())
    assert c["MAT_STRIDE"] == 136 and c["MAT_SLOTS"] == 32 and c["MAX_LAYER"] == 4096
    # The material record of the prepared tables has exactly MAT_STRIDE words.
    opts = pkg.RenderOptions(width=8, height=8)
    s = pkg.Scene.cornell()
    p = pkg.prepare(s, opts)
    off_mat, off_pl = p.params.offs0[2], p.params.offs0[3]
    assert (off_pl - off_mat) % c["MAT_STRIDE"] == 0
    assert (off_pl - off_mat) // c["MAT_STRIDE"] == 4
