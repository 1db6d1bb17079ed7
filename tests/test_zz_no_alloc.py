"""senga_rhs_noalloc, the allocation-free right-hand side, against the
context-based entry point senga_rhs_host and against the oracle.

Callers that cannot allocate device memory while they run (a host that
reserves all device memory at start-up, or one living inside another
framework's memory pool) use senga_rhs_noalloc: it takes caller-owned device
buffers and keeps its intermediates in a fixed device array inside the
library. The tests check its results on two calls in a row, that the second
call leaves the device's free memory unchanged, and that it refuses boxes
beyond the array's size. This file is named to be collected last, so a run
that stops at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

TOL = 1e-10  # same field-normalised relative L-infinity bound as the parity tests

# (case, shape or None for a 16^3 cube, z planes kept): the last one is a 2D
# box (one point in z), which the context path also accepts
CASES = [("ignition32", None, None), ("h2_kernels", None, None), ("h2_pool", (20, 14, 6), 1)]


def _case(name, shape, zkeep):
    import cases

    c = cases.make_case(name, n=None if shape else 16, seed=3, shape=shape)
    if zkeep:
        c = dict(c)
        c["fields"] = np.ascontiguousarray(c["fields"][:, :zkeep])
        c["T"] = np.ascontiguousarray(c["T"][:zkeep])
        c["itn"] = np.ascontiguousarray(c["itn"][:zkeep])
        c["shape"] = (c["shape"][0], c["shape"][1], zkeep)
    return c


@pytest.mark.parametrize("name,shape,zkeep", CASES, ids=[c[0] + ("-2d" if c[2] else "") for c in CASES])
def test_rhs_noalloc_matches_context_rhs_and_oracle_twice(name, shape, zkeep):
    import torch

    import senga
    from oracle import Oracle

    c = _case(name, shape, zkeep)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    box = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    box.upload(c["fields"], c["T"], c["itn"])
    want, t_want, _ = box.rhs()
    ref = Oracle(c["shape"], c["lengths"], c["chem"], c["diff"], c["dt"])
    ref.upload(c["fields"], c["T"], c["itn"])
    oracle_rhs, oracle_t, _ = ref.rhs()

    dev = torch.device("cuda", 0)
    state = torch.from_numpy(np.ascontiguousarray(c["fields"])).to(dev)
    t_host = torch.from_numpy(c["T"])
    i_host = torch.from_numpy(c["itn"])
    trun = torch.empty(c["T"].shape, dtype=torch.float64, device=dev)
    itn = torch.empty(c["itn"].shape, dtype=torch.int32, device=dev)
    rhs = torch.full_like(state, float("nan"))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    free_after = []
    for call in range(2):
        trun.copy_(t_host)
        itn.copy_(i_host)
        torch.cuda.synchronize(dev)
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = senga.lib.senga_rhs_noalloc(C.byref(box.cfg), C.byref(chem.t), C.byref(diff.t), state.data_ptr(),
                                         trun.data_ptr(), itn.data_ptr(), rhs.data_ptr(), status.data_ptr(), stream)
        assert rc == 0, senga.lib.senga_last_error()
        torch.cuda.synchronize(dev)
        free_after.append(torch.cuda.mem_get_info(dev)[0])
        if call == 1:
            # the array and the kernels were loaded by the first call: the
            # second one takes no device memory at all
            assert free_after[1] == free_before, (free_before, free_after[1])
        got = rhs.cpu().numpy()
        assert int(status.item()) == 0
        assert rel_linf(trun.cpu().numpy(), t_want) <= TOL, f"call {call}: T vs context"
        assert rel_linf(trun.cpu().numpy(), oracle_t) <= TOL, f"call {call}: T vs oracle"
        for k in range(want.shape[0]):
            assert rel_linf(got[k], want[k]) <= TOL, f"call {call}: field {k} vs context"
            assert rel_linf(got[k], oracle_rhs[k]) <= TOL, f"call {call}: field {k} vs oracle"
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
    # the size check comes before any device work: the pointers are never used
    rc = senga.lib.senga_rhs_noalloc(C.byref(cfg), C.byref(chem.t), C.byref(diff.t), 1, 1, 1, 1, 1, None)
    assert rc == 1
    assert b"limit" in senga.lib.senga_last_error()


def test_rhs_noalloc_requires_a_status_word():
    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    cfg = senga.ConfigT()
    cfg.nx = cfg.ny = cfg.nz = 16
    cfg.xgdlen = cfg.ygdlen = cfg.zgdlen = 1e-3
    for i in range(6):
        cfg.nend[i] = senga.NPERI
    cfg.tstep = 1e-9
    rc = senga.lib.senga_rhs_noalloc(C.byref(cfg), C.byref(chem.t), None, 1, 1, 1, 1, None, None)
    assert rc == 1
    assert b"null argument" in senga.lib.senga_last_error()


def test_rhs_noalloc_refuses_stream_capture():
    """The tables are copied from host structs at every call, so the call
    refuses a capturing stream with SENGA_ERR_UNSUPPORTED and queues
    nothing (the capture ends cleanly, with an empty graph)."""
    import warnings

    import torch

    import cases
    import senga

    chem = senga.Chem(cases.CHEM_1STEP)
    cfg = senga.ConfigT()
    cfg.nx = cfg.ny = cfg.nz = 16
    cfg.xgdlen = cfg.ygdlen = cfg.zgdlen = 1e-3
    for i in range(6):
        cfg.nend[i] = senga.NPERI
    cfg.tstep = 1e-9
    dev = torch.device("cuda", 0)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    side = torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # the empty-graph warning
        with torch.cuda.graph(g, stream=side):
            rc = senga.lib.senga_rhs_noalloc(C.byref(cfg), C.byref(chem.t), None, 1, 1, 1, 1, status.data_ptr(),
                                             side.cuda_stream)
    assert rc == 5
    assert b"captured" in senga.lib.senga_last_error()
    torch.cuda.synchronize(dev)
