"""The allocation-free optic entry point (flyb_optic_run_noalloc), called through the C ABI.

Some hosts cannot allocate device memory while they step the brain (they own every buffer, or
forbid allocation inside their step callback). For them the library keeps the optic substep's
scratch in its own file-scope device array. This checks, on two calls in a row, that the
allocation-free entry point gives what flyb_optic_run gives with caller-provided scratch, and that
requests beyond the array's stated size are refused. Collected last so that a stop at the first
failure has already run every other test; it also passes alone in a fresh process.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

from flyb200 import _abi, synthetic

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-5, 1e-6


def _args(cfg, W, state, launch, status, with_scratch):
    v, ad, pr, spk, a, b = state
    dr = torch.zeros_like(v) if with_scratch else None
    dr_tmp = torch.zeros_like(v) if with_scratch else None
    sync = torch.zeros(64, dtype=torch.int32, device="cuda") if with_scratch else None
    args = _abi.OpticArgs(m=cfg.m, batch=v.shape[1], nsteps=15, launch=launch, ptr=W[0].data_ptr(),
                          cw=W[1].data_ptr(), v=v.data_ptr(), adapt=ad.data_ptr(),
                          dr=None if dr is None else dr.data_ptr(), dr_tmp=None if dr_tmp is None else dr_tmp.data_ptr(),
                          pr=pr.data_ptr(), spk=spk.data_ptr(), a=a.data_ptr(), b=b.data_ptr(), gr=cfg.gain_rr,
                          ga=cfg.adapt_gain, aad=cfg.aad, status=status.data_ptr(),
                          sync=None if sync is None else sync.data_ptr())
    return args, (dr, dr_tmp, sync)


@pytest.mark.parametrize("launch", [_abi.LAUNCH_PERSISTENT, _abi.LAUNCH_STEP])
def test_noalloc_matches_the_allocating_entry_point_twice(launch):
    lib = _abi.lib()
    cfg = synthetic.optic_config3(seed=9, m=5000, nnz=250_000, n_pr=300, n_types=40, n_spk=400)
    Wr = cfg.W_rr()
    cw = np.stack([Wr.indices.astype(np.int32), Wr.data.astype(np.float32).view(np.int32)], axis=1)
    W = [torch.from_numpy(Wr.indptr.astype(np.int32)).cuda(), torch.from_numpy(np.ascontiguousarray(cw)).cuda()]
    rng = np.random.default_rng(4)
    B = 3
    init = [torch.from_numpy((rng.standard_normal((cfg.m, B)) * s).astype(np.float32)).cuda() for s in (0.3, 0.05, 0.3, 0.1)]
    consts = [torch.from_numpy(cfg.a).cuda(), torch.from_numpy(cfg.b).cuda()]
    ref_state = [t.clone() for t in init] + consts
    new_state = [t.clone() for t in init] + consts
    status_ref = torch.zeros(4, dtype=torch.int32, device="cuda")
    status_new = torch.zeros(4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        a_ref, keep = _args(cfg, W, ref_state, launch, status_ref, True)
        assert lib.flyb_optic_run(ct.byref(a_ref), stream) == 0
        a_new, _ = _args(cfg, W, new_state, launch, status_new, False)
        assert lib.flyb_optic_run_noalloc(ct.byref(a_new), stream) == 0
        torch.cuda.synchronize()
        assert status_ref[0].item() == 0 and status_new[0].item() == 0
        for k, name in ((0, "v"), (1, "adapt")):
            np.testing.assert_allclose(new_state[k].cpu().numpy(), ref_state[k].cpu().numpy(), rtol=RTOL, atol=ATOL,
                                       err_msg=f"{name}, call {call}")
        del keep


def test_noalloc_refuses_sizes_beyond_its_array():
    lib = _abi.lib()
    m = 1 << 20
    big = _abi.OpticArgs(m=m, batch=2, nsteps=1, launch=_abi.LAUNCH_STEP, ptr=1, v=1, adapt=1, pr=1, spk=1, a=1, b=1)
    assert lib.flyb_optic_run_noalloc(ct.byref(big), None) == _abi.ETOOBIG
