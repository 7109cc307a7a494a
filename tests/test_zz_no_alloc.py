"""The allocation-free field entry point (dct_b200_field_noalloc) against
the engine's ordinary transform, bit for bit, on two calls in a row.

It serves callers that may not allocate device memory themselves — for
instance a host framework whose caching allocator must own every buffer —
so the test hands it buffers allocated by torch, checks that the map it
writes equals the one dct_transform computes, and checks that the device's
free memory is the same before and after each checked call."""
import ctypes

import numpy as np
import pytest

from coldcore_b200.gpu import GpuBackend, load_plugin

pytestmark = pytest.mark.gpu


def _noalloc(lib, problem_id, axes, R, mu, role, cnt_t, map_t, stream):
    ax = (ctypes.c_int * len(axes))(*axes)
    return lib.dct_b200_field_noalloc(
        ctypes.c_int(problem_id), ctypes.c_int(len(axes)), ax,
        ctypes.c_int(R), ctypes.c_int(mu), ctypes.c_int(role),
        ctypes.c_void_p(cnt_t.data_ptr()), ctypes.c_void_p(map_t.data_ptr()),
        ctypes.c_longlong(stream))


@pytest.fixture(scope="module")
def warmed():
    """The first call on a device commits the library's fixed array to
    device memory (CUDA loads modules lazily) and looks up its address, so
    a caller that must not see memory move makes one small call first, as
    this fixture does; every checked call after it must leave the free
    device memory unchanged."""
    import torch
    lib = load_plugin()
    cnt = torch.zeros(9, dtype=torch.int16, device="cuda")
    out = torch.zeros(9, dtype=torch.int32, device="cuda")
    assert _noalloc(lib, 0, [3, 3], 1, 1, 0, cnt, out, 0) == 0
    torch.cuda.synchronize()
    return lib


@pytest.mark.parametrize("problem,pid,axes,R,mu", [
    ("hamming", 0, [3] * 8, 2, 1), ("hamming", 0, [2] * 12, 3, 2),
    ("lee", 2, [5, 6, 7], 2, 1), ("hamming", 0, [3] * 13, 3, 1),
    # a first group of 16-ary axes with seven layers: the tile bound
    ("hamming", 0, [16] * 4, 6, 1), ("lee", 2, [7] * 6, 4, 2)])
def test_noalloc_field_matches_transform(warmed, problem, pid, axes, R,
                                         mu):
    import torch
    lib = warmed
    rng = np.random.default_rng(11)
    size = int(np.prod(axes))
    with GpuBackend(axes, R, problem=problem, mu=mu) as b:
        stream = torch.cuda.current_stream().cuda_stream
        for call in range(2):                       # two calls in a row
            code = rng.choice(size, size=max(3, size // 60), replace=False)
            b.recount(code)
            cnt = torch.from_numpy(b.read_cnt().view(np.int16)).cuda()
            out = torch.full((size,), -7, dtype=torch.int32, device="cuda")
            role = call % 2
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info()
            assert _noalloc(lib, pid, axes, R, mu, role, cnt, out, stream) == 0
            torch.cuda.synchronize()
            free1, _ = torch.cuda.mem_get_info()
            assert free1 == free0, "the call changed the device's free memory"
            (b.gain_map if role == 0 else b.loss_map)()
            assert np.array_equal(out.cpu().numpy(), b.map_all())


def test_noalloc_rejects_cells_beyond_its_array():
    import torch
    lib = load_plugin()
    cnt = torch.zeros(8, dtype=torch.int16, device="cuda")
    out = torch.zeros(8, dtype=torch.int32, device="cuda")
    # 3^16 words x 5 layers is more than the fixed 16M-word array
    assert _noalloc(lib, 0, [3] * 16, 4, 1, 0, cnt, out, 0) == -6
