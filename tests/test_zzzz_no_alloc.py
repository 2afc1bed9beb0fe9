"""cismgpu_global_sum_stagger_noalloc: the owned-vertex global sum with caller-owned device
buffers and library-internal fixed scratch, called through the C ABI.

Its results must equal the allocating entry point's (cismgpu_global_sum_stagger) bit for
bit -- the tolerance every global-sum test here uses -- on two calls in a row on one
stream (the second one reusing the shared scratch the first one left behind).  The file
is named to be collected last, and also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import cism_b200 as cg
from cism_b200 import assembly as asm

pytestmark = pytest.mark.gpu


def fields(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    a1 = rng.standard_normal((ny - 1, nx - 1, nz)) * np.exp(rng.uniform(-20, 20, (ny - 1, nx - 1, nz)))
    a2 = rng.standard_normal((ny - 1, nx - 1, nz))
    return a1, a2


CASES = [(37, 29, 11, "periodic"), (1001, 803, 1, "no_ice"), (260, 190, 7, "outflow")]


@pytest.mark.parametrize("nx,ny,nz,bc", CASES, ids=[f"{c[0]}x{c[1]}x{c[2]}-{c[3]}" for c in CASES])
def test_noalloc_matches_allocating_entry_two_calls(gpu_lib, nx, ny, nz, bc):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    par = asm.default_par(nx, ny, bc)
    inputs = [fields(nx, ny, nz, seed) for seed in (nz, nz + 100)]
    d_in = [(torch.from_numpy(a1).to(dev), torch.from_numpy(a2).to(dev)) for a1, a2 in inputs]
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    for c, (t1, t2) in enumerate(d_in):      # two calls in a row, same stream, no sync between
        cg.parallel_global_sum_stagger_noalloc(nx, ny, nz, par, t1.data_ptr(), t2.data_ptr(),
                                               out[c:].data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    got = out.cpu().numpy()
    for c, (a1, a2) in enumerate(inputs):
        want = cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, a2)
        assert got[c] == want, (c, got[c], want)


def test_noalloc_rejects_oversized_and_host_buffers(gpu_lib):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    t = torch.zeros(64, dtype=torch.float64, device=dev)
    # (nx-1)*(ny-1) just over the limit: rejected before anything is enqueued
    nx, ny = 2049, 2050
    assert (nx - 1) * (ny - 1) == cg.NOALLOC_MAX_COLUMNS + 2048
    with pytest.raises(cg.CismGpuError) as e:
        cg.parallel_global_sum_stagger_noalloc(nx, ny, 1, asm.default_par(nx, ny, "periodic"), t.data_ptr(),
                                               t.data_ptr(), t.data_ptr(), 0)
    assert e.value.status == 4 and "limit" in str(e.value)
    # a pageable host array is not device-accessible: rejected by the pointer check
    host = np.zeros((7, 7, 1))
    with pytest.raises(cg.CismGpuError) as e:
        cg.parallel_global_sum_stagger_noalloc(8, 8, 1, asm.default_par(8, 8, "periodic"),
                                               host.ctypes.data_as(ctypes.c_void_p).value, t.data_ptr(),
                                               t.data_ptr(), 0)
    assert e.value.status == 4
    # parallel%reprosum needs host steps between its kernels: rejected, not summed another way
    with pytest.raises(cg.CismGpuError) as e:
        cg.parallel_global_sum_stagger_noalloc(8, 8, 1, dict(asm.default_par(8, 8, "periodic"), reprosum=1),
                                               t.data_ptr(), t.data_ptr(), t.data_ptr(), 0)
    assert e.value.status == 3 and "reprosum" in str(e.value)
    # more than one task: the whole domain must be on this GPU
    with pytest.raises(cg.CismGpuError) as e:
        cg.parallel_global_sum_stagger_noalloc(8, 8, 1, dict(asm.default_par(8, 8, "periodic"), tasks_col=2),
                                               t.data_ptr(), t.data_ptr(), t.data_ptr(), 0)
    assert e.value.status == 3
    torch.cuda.synchronize(dev)
