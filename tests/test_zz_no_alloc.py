"""dmpm_compute_volumes_noalloc: particle volumes for callers that cannot
allocate device memory (a frame loop that must not take cudaMalloc's
device-wide synchronisation, or a process whose device memory is held by
another allocator).  The test allocates the caller's buffers itself (with
torch) and checks the no-allocation entry point against the context-based
dmpm_compute_volumes on two calls in a row: the second call must not see the
first call's masses left in the shared scratch array.  It is collected last
so that a run stopping at the first failure has already run everything else,
and it passes alone in a fresh process as well."""
import ctypes

import numpy as np
import pytest

import dmpm
import scenes
from tests.helpers import relerr

pytestmark = pytest.mark.gpu


def _volumes_via_context(sc):
    with dmpm.Context("fp32") as c:
        c.set_grid(sc.dims, sc.dx, sc.min_point)
        c.set_particles(sc.x, sc.m, sc.lam, sc.mu)
        c.compute_volumes()
        c.set_params(dt=1e-4)
        c.setup(1)
        return c.get(0, "vol")


def test_noalloc_volumes_match_context_path_twice(gpu_ready):
    import torch

    lib = dmpm.load_library()
    sc = scenes.small_scene(seed=31, res=48, radius=0.3)
    want = _volumes_via_context(sc)
    x = torch.tensor(sc.x, dtype=torch.float32, device="cuda").contiguous()
    m = torch.tensor(sc.m, dtype=torch.float32, device="cuda")
    mn = (ctypes.c_float * 3)(*[float(v) for v in sc.min_point])
    stream = torch.cuda.current_stream().cuda_stream
    vols = [torch.full((sc.n,), -1.0, dtype=torch.float32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for call in range(2):
        vol = vols[call]
        # the device's free memory (cudaMemGetInfo) must not move across a call after the first
        free_before = torch.cuda.mem_get_info()[0]
        st = lib.dmpm_compute_volumes_noalloc(sc.n, x.data_ptr(), m.data_ptr(), sc.dims[0], sc.dims[1], sc.dims[2],
                                             float(sc.dx), mn, vol.data_ptr(), stream)
        assert st == dmpm.OK, call
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        got = vol.cpu().numpy().astype(np.float64)
        assert relerr(got, want) < 1e-5, call


def test_noalloc_rejects_grids_beyond_capacity(gpu_ready):
    lib = dmpm.load_library()
    mn = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
    # 102^3 = 1,061,208 nodes > 1,048,576: rejected before any GPU work
    st = lib.dmpm_compute_volumes_noalloc(0, None, None, 102, 102, 102, 1.0, mn, None, None)
    assert st == dmpm.ERR_TOO_LARGE
    st = lib.dmpm_compute_volumes_noalloc(0, None, None, 101, 101, 101, 1.0, mn, None, None)
    assert st == dmpm.OK
