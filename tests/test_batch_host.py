"""Host-side batch tables (no GPU): tile numbering, pixel and Gaussian bases."""
from __future__ import annotations

import torch

from structsplat_b200.batch import Batch, FitSettings


def test_batch_tables_number_tiles_image_by_image():
    sizes, counts = [(64, 96), (37, 50), (1, 1), (0, 5)], [5, 0, 2, 1]
    b = Batch(sizes, counts, tile_size=32, device="cpu")
    assert b.images == 4
    # tiles: 3x2, 2x2, 1x1, 1x0
    assert b.image_table.tolist() == [[64, 96, 3, 0], [37, 50, 2, 6], [1, 1, 1, 10],
                                      [0, 5, 1, 11]]
    assert b.tiles == 11 and b.pixels == 64 * 96 + 37 * 50 + 1
    assert b.pixel_base.tolist() == [0, 6144, 6144 + 1850, 6144 + 1850 + 1]
    assert b.gaussian_base.tolist() == [0, 5, 5, 7, 8]
    assert b.gaussian_image.tolist() == [0, 0, 0, 0, 0, 2, 2, 3]
    assert b.tile_image.tolist() == [0] * 6 + [1] * 4 + [2]
    flat = torch.arange(b.pixels * 3, dtype=torch.float32).view(-1, 3)
    parts = b.split_images(flat)
    assert [tuple(p.shape) for p in parts] == [(64, 96, 3), (37, 50, 3), (1, 1, 3), (0, 5, 3)]
    assert torch.equal(b.concat_images(parts), flat)


def test_fit_settings_learning_rates():
    s = FitSettings()
    assert s.lrs() == [5e-2, 3e-2, 1e-2, 3e-2, 1e-2]  # config.py:194-198
    assert FitSettings.uniform_lr(1e-2).lrs() == [1e-2] * 5
