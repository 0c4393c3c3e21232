"""The placement oracle reproduces the reference's density, sampler and field build exactly.

Fixtures (tests/golden/pl_*) come from the reference's own density_from_energy,
sample_candidates (numpy Generator seeded) and build_field (density_random sampler).  The
sampler restatement takes explicit uniforms; drawing them from default_rng(seed) as
random(n) then random((n, 2)) reproduces the reference's points bit for bit, which pins how
Generator.choice consumes its uniforms.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_names
from oracle import placement_ref as P


@pytest.mark.parametrize("name", golden_names("pl_density_"))
def test_density_from_energy_matches_reference(name):
    z = golden(name)
    got = P.density_from_energy(z["energy"], float(z["base"]), float(z["power"]),
                                float(z["ref"]))
    assert np.array_equal(got, z["density"])


def test_energy_reference_matches_structure_tensor():
    z = golden("pl_field_aniso_onedge.npz")
    assert P.energy_reference(z["energy"]) == float(z["energy_ref"])


@pytest.mark.parametrize("name", golden_names("pl_sample_"))
def test_sampler_with_explicit_uniforms_matches_reference(name):
    z = golden(name)
    n = int(z["n"])
    pts, idx = P.sample_candidates(z["density"], n, P.uniforms_for(int(z["seed"]), n))
    assert np.array_equal(pts, z["points"])
    H, W = z["density"].shape
    assert idx.min() >= 0 and idx.max() < H * W


@pytest.mark.parametrize("name", golden_names("pl_field_"))
def test_place_field_matches_reference_build_field(name):
    z = golden(name)
    n = int(z["n"])
    pts, _ = P.sample_candidates(z["density"], n, P.uniforms_for(int(z["seed"]), n))
    f = P.place_field(z["img"], z["density"], z["angle"], z["coherence"], pts, n,
                      anisotropic=bool(z["anisotropic"]))
    for k in ("means", "log_scales", "rotations", "colors"):
        assert np.array_equal(f[k], z[k]), k
