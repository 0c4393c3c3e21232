"""TEST INFRASTRUCTURE ONLY — the CPU oracle for the StructSplat tiled rasterizer path.

This package restates, on the CPU, the reference algorithm of intrinsicD/structsplat for the
hot path the CUDA library implements (file:line citations are to the reference project):

* ``render_ref``       — clipped-support normalized / additive renderer and its autograd
                         gradients (``src/structsplat/render.py:62-235``), in float32 or float64;
* ``field_ref``        — RS parameterisation → conic, 3σ radii, opacity
                         (``src/structsplat/gaussians.py:270-321``);
* ``tile_index_ref``   — the (tile → Gaussian ids) index (``src/structsplat/cuda_render.py:177-226``);
* ``structure_tensor_ref`` — ``J = G_ρ * (∇I∇Iᵀ)`` and its eigen-analysis
                         (``src/structsplat/structure_tensor.py:30-186``);
* ``ss_oracle.c`` / ``c_oracle`` — a plain-C restatement: int64 support rectangles and tile
                         index, and a float64 forward/backward used as the FP64 error yardstick
                         at full benchmark sizes.

It is pinned against golden vectors generated from the reference itself
(``tests/golden/make_golden.py``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` may import it, and only as the checker or the timed CPU
baseline.  The product package ``structsplat_b200`` never imports it and has no CPU fallback.
"""
