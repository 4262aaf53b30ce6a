"""mpp_volume_noalloc: the liquid volume for callers that cannot allocate device memory.

A caller such as a monitoring or render callback working under a fixed memory budget
cannot create a solver context (that allocates the whole workspace) just to read the
volume. mpp_volume_noalloc runs the volume reduction with its scratch in a static device
array instead. These checks call it through the C ABI and compare it with the context
entry point, mpp_volume, within the volume tolerance the other tests use, on two calls
in a row (the shared scratch must not carry anything from one call into the next).

This file is collected last on purpose: it must pass after every other test in the same
process as well as alone in a fresh one.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VOLUME_RTOL = 1e-6


def _noalloc(lib, grid, phi, stream):
    from mpp import grid_struct

    out = ctypes.c_double(-1.0)
    g = grid_struct(grid)
    code = lib.mpp_volume_noalloc(ctypes.byref(g), ctypes.c_void_p(phi.data_ptr()), ctypes.byref(out),
                                  ctypes.c_void_p(stream.cuda_stream))
    return code, out.value


def test_noalloc_volume_matches_context(cuda):
    import torch

    import mpp
    from mpp import _lib, scene

    lib = _lib.load()
    stream = torch.cuda.current_stream(cuda)
    # 64^3, then the largest grid the scratch admits (256^3 = 16,777,216 cells), then a
    # different 64^3 basin: three calls in a row on the shared scratch.
    basins = [scene.box_basin(64, seed=1064), scene.config_basin("whirl256"),
              scene.box_basin(64, seed=7, height=0.35, wall=0.4)]
    for basin in basins:
        phi = torch.from_numpy(basin.phi).to(cuda)
        want = mpp.Projector(basin.grid).volume(phi)
        for _ in range(2):
            code, got = _noalloc(lib, basin.grid, phi, stream)
            assert code == 0, _lib.last_error()
            assert abs(got - want) <= VOLUME_RTOL * abs(want), (basin.name, got, want)


def test_noalloc_volume_rejects_oversize_grid(cuda):
    import torch

    from mpp import _lib, scene

    lib = _lib.load()
    grid = scene.Grid(lo=(0.0, 0.0, 0.0), dx=0.05, n=(258, 256, 256), radius=5.0, floor=0.0, levels=2)
    phi = torch.zeros(16, dtype=torch.float32, device=cuda)  # never read: the size is refused first
    code, _ = _noalloc(lib, grid, phi, torch.cuda.current_stream(cuda))
    assert code == _lib.ERR_INVALID
    assert "at most 16777216 cells" in _lib.last_error()
