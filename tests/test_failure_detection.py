"""Failure detection of the device-side bounded waits, without a GPU fault.

Every step kernel waits on mbarriers for its TMA loads with a poll limit; on
giving up it sets the workspace status word to GB_E_TIMEOUT and returns, and
gb_workspace_status reports it.  gb_selftest_bounded_wait runs that wait on
an mbarrier that nothing completes (a second arrival that is never made), so
the timeout path runs for real, with a short limit, and the context must
stay usable afterwards."""
import time

import numpy as np
import pytest
import torch

from conftest import load_case, oracle_kwargs
from geobrain_b200 import _lib
from oracle import oracle as orc


def test_selftest_argument_checks_need_no_gpu():
    lib = _lib.load()
    assert lib.gb_selftest_bounded_wait(None, 0, 0, 10, None) == _lib.GB_E_ARG
    assert lib.gb_selftest_bounded_wait(4096, 0, 0, 10, None) == _lib.GB_E_WORKSPACE
    assert lib.gb_selftest_bounded_wait(4096, 1024, 0, 0, None) == _lib.GB_E_ARG
    assert lib.gb_selftest_bounded_wait(4096, 1024, 0, (1 << 22) + 1, None) == _lib.GB_E_ARG


@pytest.mark.gpu
def test_wait_that_never_completes_reports_timeout_and_context_survives(cuda_device):
    lib = _lib.load()
    ws = torch.zeros(1024, dtype=torch.uint8, device=cuda_device)
    st = torch.cuda.current_stream(cuda_device).cuda_stream
    assert lib.gb_selftest_bounded_wait(ws.data_ptr(), ws.numel(), 1, 1000, st) == _lib.GB_OK
    t0 = time.perf_counter()
    rc = lib.gb_selftest_bounded_wait(ws.data_ptr(), ws.numel(), 0, 20000, st)
    elapsed = time.perf_counter() - t0
    assert rc == _lib.GB_E_TIMEOUT, rc
    assert b"timed out" in lib.gb_last_error()
    assert elapsed < 10.0, elapsed
    # the status word is re-armed by the next call, and the wait completes again
    assert lib.gb_selftest_bounded_wait(ws.data_ptr(), ws.numel(), 1, 1000, st) == _lib.GB_OK

    # the CUDA context is intact: a forward right after matches the oracle
    from geobrain_b200.wave import acoustic_forward_kernel
    c = load_case("small_nofs")
    out = acoustic_forward_kernel(
        nx=c["nx"], nz=c["nz"], dx=c["dx"], dz=c["dx"], nt=c["nt"], dt=c["dt"], nabc=c["nabc"],
        free_surface=False, src_x=c["src_x"], src_z=c["src_z"], src_n=len(c["src_x"]),
        src_v=torch.as_tensor(c["src_v"], device=cuda_device), rcv_x=c["rcv_x"], rcv_z=c["rcv_z"],
        rcv_n=len(c["rcv_x"]), damp=torch.as_tensor(c["damp"], device=cuda_device),
        vp=torch.as_tensor(c["vp"], device=cuda_device), rho=torch.as_tensor(c["rho"], device=cuda_device),
        device=cuda_device)
    ref = orc.forward(**oracle_kwargs(c), half=2, dtype=np.float64)
    assert orc.rel_l2(out["p"].cpu().numpy(), ref["p"]) < 1e-5
