"""Placement on the GPU against the reference's density, sampler and field build.

Fixtures (tests/golden/pl_*) are the reference's own outputs.  Bars: the density pmf within
1e-13 relative (only the order of the float64 sum differs); sampled points bit-identical given
the reference's uniforms (the pixel choice is a search in the float64 cdf, whose parallel prefix
sum differs from numpy's serial one only in the last bits); the field at given points
bit-identical except log-scales (CUDA logf vs torch's CPU log: 2 ulp).  End to end, with the
GPU structure tensor in front (float32 parity ~1e-6), at least 99% of the points and their
fields match.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import require_cuda
from oracle import placement_ref as P
from structsplat_b200 import placement as PL
from structsplat_b200 import structure_tensor as st

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names("pl_density_"))
def test_density_matches_reference(name):
    require_cuda()
    z = golden(name)
    got = PL.density_from_energy(torch.tensor(z["energy"], device="cuda"), float(z["base"]),
                                 float(z["power"]), ref=float(z["ref"])).cpu().numpy()
    want = z["density"]
    assert np.max(np.abs(got - want) / np.maximum(want, 1e-300)) <= 1e-13


def test_energy_reference_on_device_matches_reference():
    require_cuda()
    z = golden("pl_field_aniso_onedge.npz")
    got = float(PL.energy_reference(torch.tensor(z["energy"], device="cuda"))[0])
    assert abs(got - float(z["energy_ref"])) <= 1e-15 * float(z["energy_ref"])


@pytest.mark.parametrize("name", golden_names("pl_sample_"))
def test_sampler_matches_reference_points(name):
    require_cuda()
    z = golden(name)
    n = int(z["n"])
    dens = torch.tensor(z["density"], device="cuda")
    pts = PL.sample_candidates(dens, n, rng=np.random.default_rng(int(z["seed"])))
    assert np.array_equal(pts.cpu().numpy(), z["points"])


def test_sampler_edge_cases():
    require_cuda()
    # a single pixel with all the mass: every point lands within half a pixel of it, reflected
    d = torch.zeros(5, 6, dtype=torch.float64, device="cuda")
    d[0, 5] = 1.0
    pts, idx = PL.sample_candidates(d, 1000, generator=torch.Generator("cuda").manual_seed(0),
                                    return_index=True)
    assert torch.all(idx == 5)
    p = pts.cpu().numpy()
    assert np.all(p[:, 0] <= 5.0) and np.all(p[:, 0] >= 4.5)
    assert np.all(p[:, 1] >= 0.0) and np.all(p[:, 1] <= 0.5)
    # zero samples
    assert PL.sample_candidates(d, 0, generator=torch.Generator("cuda")).shape == (0, 2)


@pytest.mark.parametrize("name", golden_names("pl_field_"))
def test_field_at_reference_points_matches_build_field(name):
    require_cuda()
    z = golden(name)
    n = int(z["n"])
    pts, _ = P.sample_candidates(z["density"], n, P.uniforms_for(int(z["seed"]), n))
    tensor = st.StructureTensor(None, None, torch.tensor(z["angle"], device="cuda"),
                                torch.tensor(z["coherence"], device="cuda"), None, None)
    f = PL.field_at_points(torch.tensor(z["img"], device="cuda"),
                           torch.tensor(z["density"], device="cuda"), tensor,
                           torch.tensor(pts, device="cuda"), n,
                           anisotropic=bool(z["anisotropic"]))
    for k in ("means", "rotations", "colors"):
        assert np.array_equal(f[k].cpu().numpy(), z[k]), k
    ls = f["log_scales"].cpu().numpy()
    assert np.max(np.abs(ls - z["log_scales"]) / np.maximum(np.abs(z["log_scales"]), 1e-3)) <= 3e-7


@pytest.mark.parametrize("name", golden_names("pl_field_"))
def test_place_field_end_to_end_matches_reference(name):
    require_cuda()
    z = golden(name)
    n = int(z["n"])
    strategy = "aniso_onedge" if int(z["anisotropic"]) else "iso_blue_noise"
    f, _, _ = PL.place_field(torch.tensor(z["img"], device="cuda"), n, strategy=strategy,
                             seed=int(z["seed"]))
    same = np.all(f["means"].cpu().numpy() == z["means"], axis=1)
    assert same.mean() >= 0.99
    for k, tol in (("rotations", 1e-5), ("colors", 1e-6), ("log_scales", 1e-5)):
        got = f[k].cpu().numpy()[same]
        want = z[k][same]
        assert np.max(np.abs(got - want)) <= tol * max(1.0, np.abs(want).max()), k
