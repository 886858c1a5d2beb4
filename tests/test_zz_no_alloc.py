"""emma_hydro_level_dt_noalloc: the level time step from a level state already
on the device, with the reduction's scratch in a fixed array of the library
(no cudaMalloc).  Its dt must equal emma_hydro_comptstep's for the same state,
on consecutive calls that reuse the scratch (a large level, then smaller and
slower ones: stale partial maxima of the first call must not leak into the
next).  Collected last so that it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

from emma_b200 import configs, PREC_FP64, ResidentHydro
from emma_b200._lib import lib, ST_ARG

CFL = 0.8
MAX_CELLS = 33554432


def noalloc_dt(d_state, ncells, level, stream=None):
    dt = ctypes.c_double(-1.0)
    st = lib().emma_hydro_level_dt_noalloc(d_state, ncells, level, CFL, stream, ctypes.byref(dt))
    return st, dt.value


def check_level(r, level, scale=1.0):
    """Scale the level's speeds by `scale`, then compare both entries' dt."""
    import torch
    st = r.state(level)
    if scale != 1.0:
        st[1:4] *= scale
        st[4] *= scale * scale
        r.set_state(level, st)
    ref = r.comptstep(level)
    dev = torch.from_numpy(np.ascontiguousarray(st)).cuda()
    torch.cuda.synchronize()
    code, dt = noalloc_dt(dev.data_ptr(), st.shape[1], level, torch.cuda.current_stream().cuda_stream)
    assert code == 0
    # a maximum is exact and both entries round the signal speed identically
    assert dt > 0 and dt == ref, (level, dt, ref)
    return dt


@pytest.mark.gpu
def test_noalloc_dt_matches_comptstep(gpu):
    # call 1: a 128^3 level (1024 reduction blocks), speeds raised x4
    big = configs.random_uniform(level=7)
    r = ResidentHydro(big.build(), precision=PREC_FP64, cfl=CFL)
    dt1 = check_level(r, 7, scale=4.0)
    # call 2 right after on the same level state at lower speed: same block count
    dt2 = check_level(r, 7, scale=0.25)
    assert dt2 > dt1
    # calls 3..5: a smaller tree whose levels need far fewer blocks, slower again
    amr = configs.small_amr()
    r = ResidentHydro(amr.build(), precision=PREC_FP64, cfl=CFL)
    for level in range(amr.lcoarse, amr.lmax + 1):
        assert check_level(r, level, scale=0.5) > 0


@pytest.mark.gpu
def test_noalloc_dt_limits(gpu):
    import torch
    dev = torch.zeros(8, dtype=torch.float64, device="cuda")
    code, dt = noalloc_dt(dev.data_ptr(), 0, 5)
    assert code == 0 and dt == 1e9
    code, _ = noalloc_dt(dev.data_ptr(), MAX_CELLS + 1, 5)
    assert code == ST_ARG
    # after the cached scratch addresses are dropped, the next call looks its address up again
    lib().emma_hydro_noalloc_forget()
    code, dt = noalloc_dt(dev.data_ptr(), 0, 5)
    assert code == 0 and dt == 1e9


def test_noalloc_rejects_arguments_on_host():
    """Rejections happen before any CUDA call (no GPU needed)."""
    fake = ctypes.c_void_p(256)  # never dereferenced: every case below is refused first
    assert noalloc_dt(None, 8, 5)[0] == ST_ARG
    assert noalloc_dt(fake, -1, 5)[0] == ST_ARG
    assert noalloc_dt(fake, MAX_CELLS + 1, 5)[0] == ST_ARG
    assert noalloc_dt(fake, 8, 0)[0] == ST_ARG
