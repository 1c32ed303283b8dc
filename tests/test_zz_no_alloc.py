"""p3m_cell_lists_static — cell lists for callers that cannot allocate.

Some callers cannot call cudaMalloc where they need cell lists (code inside a
frame or a captured region, hosts whose device memory belongs to another
runtime such as a JVM). p3m_cell_lists_static builds the lists from and into
device arrays the caller owns, keeping its working memory in an array
compiled into the library. This test calls it through the C-ABI on device
arrays (torch tensors as plain device memory) and checks it against the
context entry point p3m_build_cell_lists on two calls in a row of different
sizes, so that anything the shared working array kept from the first call
would show in the second. The file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest

from gravity_b200 import _abi
from gravity_b200.pipeline import GravityPipeline

from helpers import clustered, small_torus

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _static_lists(sc):
    import torch

    lib = _abi.load()
    g = sc.config.gravity
    n, P = sc.n, g.grid_width * g.grid_height
    dev = torch.device("cuda", 0)
    bodies = torch.from_numpy(np.ascontiguousarray(sc.bodies)).to(dev)
    mats = torch.from_numpy(np.ascontiguousarray(sc.materials)).to(dev)
    keys = torch.full((n,), -1, dtype=torch.int32, device=dev)
    ids = torch.full((n,), -1, dtype=torch.int32, device=dev)
    start = torch.full((P,), -7, dtype=torch.int32, device=dev)
    count = torch.full((P,), -7, dtype=torch.int32, device=dev)
    mass = torch.full((P,), -7, dtype=torch.int32, device=dev)
    entries = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = lib.p3m_cell_lists_static(_ptr(bodies), _ptr(mats), n, g.grid_width, g.grid_height,
                                   _ptr(keys), _ptr(ids), _ptr(start), _ptr(count), _ptr(mass),
                                   _ptr(entries), ctypes.c_void_p(stream.cuda_stream))
    assert rc == _abi.P3M_OK, lib.p3m_last_error(None).decode()
    torch.cuda.synchronize(dev)
    return (keys.cpu().numpy().view(np.uint32), ids.cpu().numpy(), start.cpu().numpy(),
            count.cpu().numpy(), mass.cpu().numpy().view(np.uint32), entries.cpu().numpy())


def _context_lists(sc):
    with GravityPipeline(sc.config) as gpu:
        gpu.upload(sc.bodies, sc.materials)
        gpu.build_cell_lists(sc.n)
        return gpu.cell_lists(sc.n)


def _check(sc):
    sk, si, ss, sn, sm, se = _static_lists(sc)
    ck, ci, cs, cn, cm = _context_lists(sc)
    np.testing.assert_array_equal(sk, ck)
    np.testing.assert_array_equal(si, ci)
    np.testing.assert_array_equal(sn, cn)
    np.testing.assert_array_equal(sm, cm)
    occupied = cn > 0
    np.testing.assert_array_equal(ss[occupied], cs[occupied])
    # entries: (x, y, mass, ID bits) of the bodies in list order
    expect = np.empty((sc.n, 4), np.float32)
    expect[:, 0] = sc.bodies[ci, 0]
    expect[:, 1] = sc.bodies[ci, 1]
    expect[:, 2] = sc.materials[ci, 0]
    expect[:, 3] = ci.astype(np.uint32).view(np.float32)
    np.testing.assert_array_equal(se.view(np.uint32), expect.view(np.uint32))


def test_static_cell_lists_match_context_entry_point_twice(cuda_device):
    # First call: a large clustered scene; second: a smaller one on another
    # grid. Both must equal the allocating entry point's lists exactly.
    _check(clustered(n=60_000, grid=(256, 128), seed=21))
    _check(small_torus(n=7_000, grid=(128, 64), seed=22))


def test_static_cell_lists_reject_sizes_beyond_the_limit(cuda_device):
    lib = _abi.load()
    too_many = _abi.CELL_LISTS_STATIC_MAX_BODIES + 1
    dummy = ctypes.c_void_p(16)
    rc = lib.p3m_cell_lists_static(dummy, dummy, too_many, 64, 32, dummy, dummy, dummy, dummy,
                                   dummy, dummy, None)
    assert rc == _abi.P3M_ERR_CAPACITY
    assert b"at most 1048576" in lib.p3m_last_error(None)
