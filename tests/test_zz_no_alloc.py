"""The allocation-free tile index build gives exactly the index of the workspace-based build.

``ss_build_tile_index_static`` exists for callers that cannot allocate device memory while
they build a tile index (an engine that owns all device memory through its own pool, a plugin
that may only use the buffers it is handed, or code that must avoid the device synchronisation
an allocation implies).  It keeps its scratch in a fixed device array inside the library.  This
test calls it through the C ABI twice in a row, with different fields, and checks each result
against ``ss_build_tile_index`` (which takes a caller-allocated workspace) on the same inputs.
The index is integer data, so the comparison is exact.

The file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes

import pytest
import torch

from structsplat_b200 import _native
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu

_P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _field(H, W, n, seed):
    from oracle import field_ref
    f = make_field(H, W, n, seed=seed, log_sigma_std=0.8)
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    means = torch.tensor(f.means).cuda()
    conics = field_ref.conics(ls, rot).cuda().contiguous()
    radii = field_ref.radii(ls, rot, 3.0).cuda().contiguous()
    return means, conics, radii


def _with_workspace(means, conics, radii, H, W, ts, cap):
    lib = _native.lib()
    n = means.shape[0]
    T = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
    size = ctypes.c_size_t(0)
    assert lib.ss_reference_workspace_bytes(n, H, W, ts, cap, ctypes.byref(size)) == 0
    ws = torch.empty(max(size.value, 1), dtype=torch.uint8, device="cuda")
    offsets = torch.empty(T + 1, dtype=torch.int32, device="cuda")
    gids = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.ss_build_tile_index(_P(means), _P(conics), _P(radii), n, H, W, ts, 0,
                                 ctypes.c_float(3.0), _P(gids), cap, _P(offsets), _P(ws),
                                 size.value, _P(status), _stream())
    assert rc == 0, lib.ss_last_error().decode()
    return gids, offsets, status


def _static(means, conics, radii, H, W, ts, cap):
    lib = _native.lib()
    n = means.shape[0]
    T = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
    offsets = torch.empty(T + 1, dtype=torch.int32, device="cuda")
    gids = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.ss_build_tile_index_static(_P(means), _P(conics), _P(radii), n, H, W, ts, 0,
                                        ctypes.c_float(3.0), _P(gids), cap, _P(offsets),
                                        _P(status), _stream())
    assert rc == 0, lib.ss_last_error().decode()
    return gids, offsets, status


@pytest.mark.parametrize("shape", [(96, 130, 900, 3, 16), (200, 160, 2500, 4, 8)])
def test_static_index_matches_workspace_index_on_consecutive_calls(shape):
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    H, W, n, seed, ts = shape
    fields = [_field(H, W, n, seed), _field(H, W, n // 2, seed + 1)]
    for means, conics, radii in fields:  # two calls in a row share the static scratch
        cap = 64 * n
        g_ref, o_ref, s_ref = _with_workspace(means, conics, radii, H, W, ts, cap)
        g_st, o_st, s_st = _static(means, conics, radii, H, W, ts, cap)
        torch.cuda.synchronize()
        total = int(o_ref[-1])
        assert 0 < total <= cap
        assert torch.equal(o_st, o_ref)
        assert torch.equal(g_st[:total], g_ref[:total])
        assert int(s_ref.item()) == 0 and int(s_st.item()) == 0


def test_static_index_rejects_sizes_beyond_its_scratch():
    lib = _native.lib()
    size_ok = lib.ss_build_tile_index_static(None, None, None, 70000, 64, 64, 16, 0,
                                             ctypes.c_float(3.0), None, 0, None, None, None)
    assert size_ok == 2 and b"at most" in lib.ss_last_error()
    too_many_tiles = lib.ss_build_tile_index_static(None, None, None, 10, 4096, 4096, 16, 0,
                                                    ctypes.c_float(3.0), None, 0, None, None,
                                                    None)
    assert too_many_tiles == 2 and b"tiles" in lib.ss_last_error()
