"""The SSPL1 decode oracle reproduces the reference's decode (fixtures codec_*)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_names
from oracle import codec_ref

CASES = golden_names("codec_")


@pytest.mark.parametrize("name", CASES)
def test_decode_matches_reference(name):
    z = golden(name)
    d = codec_ref.decode(z["blob"].tobytes())
    for k in ("means", "log_scales", "rotations", "colors"):
        assert np.array_equal(d[k], z[k]), k
    assert ("opacity_logits" in d) == ("opacity_logits" in z.files)
    if "opacity_logits" in d:
        assert np.array_equal(d["opacity_logits"], z["opacity_logits"])


def test_fixture_inventory():
    assert len(CASES) == 3
