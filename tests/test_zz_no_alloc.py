"""senga_rhs_noalloc, the allocation-free right-hand side, against the
context-based entry point senga_rhs_host.

Callers that cannot allocate device memory while they run (a host that
reserves all device memory at start-up, or one living inside another
framework's memory pool) use senga_rhs_noalloc: it takes caller-owned device
buffers and keeps its intermediates in a fixed device array inside the
library. This file is named to be collected last, so a run that stops at the
first failure has already run every other test; it also passes on its own in
a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-10  # same field-normalised relative L-infinity bound as the parity tests


@pytest.mark.parametrize("name", ["ignition32", "h2_kernels"])
def test_rhs_noalloc_matches_context_rhs_twice(name):
    import torch

    import cases
    import senga

    c = cases.make_case(name, n=16, seed=3)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    want, t_want, _ = box.rhs()

    dev = torch.device("cuda", 0)
    state = torch.from_numpy(np.ascontiguousarray(c["fields"])).to(dev)
    trun = torch.empty(c["T"].shape, dtype=torch.float64, device=dev)
    itn = torch.empty(c["itn"].shape, dtype=torch.int32, device=dev)
    rhs = torch.full_like(state, float("nan"))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        trun.copy_(torch.from_numpy(c["T"]))
        itn.copy_(torch.from_numpy(c["itn"]))
        rc = senga.lib.senga_rhs_noalloc(C.byref(box.cfg), C.byref(chem.t), C.byref(diff.t), state.data_ptr(),
                                         trun.data_ptr(), itn.data_ptr(), rhs.data_ptr(), status.data_ptr(), stream)
        assert rc == 0, senga.lib.senga_last_error()
        torch.cuda.synchronize(dev)
        got = rhs.cpu().numpy()
        assert int(status.item()) == 0
        assert rel_linf(trun.cpu().numpy(), t_want) <= TOL, f"call {call}: T"
        for k in range(want.shape[0]):
            assert rel_linf(got[k], want[k]) <= TOL, f"call {call}: field {k}"
        rhs.fill_(float("nan"))


def test_rhs_noalloc_rejects_boxes_beyond_the_scratch_limit():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_H2)
    diff = senga.Diff(cases.DIFF_H2, chem)
    cfg = senga.ConfigT()
    cfg.nx = cfg.ny = cfg.nz = 64  # 262,144 points x 50 doubles > 16 MiB
    cfg.xgdlen = cfg.ygdlen = cfg.zgdlen = 1e-3
    for i in range(6):
        cfg.nend[i] = senga.NPERI
    cfg.tstep = 1e-9
    rc = senga.lib.senga_rhs_noalloc(C.byref(cfg), C.byref(chem.t), C.byref(diff.t), 1, 1, 1, 1, None, None)
    assert rc == 1
    assert b"limit" in senga.lib.senga_last_error()
