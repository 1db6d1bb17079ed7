"""Stream-ordered upload/download (senga_upload_state_async,
senga_download_state_async): two contexts fed alternately from page-locked
host buffers give bit-identical results to the synchronous host calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_async_copies_on_two_contexts_match_the_synchronous_path():
    import torch

    import cases
    import senga

    c = cases.make_case("h2_kernels", n=16, seed=51)
    chem = senga.Chem(c["chem"])
    diff = senga.Diff(c["diff"], chem)
    ref = senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"])
    ref.upload(c["fields"], c["T"], c["itn"])
    ref.step(1, graph=True)
    want = ref.download()

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out

    src = tuple(pinned(np.ascontiguousarray(a)) for a in (c["fields"], c["T"], c["itn"].astype(np.int32)))
    boxes = [senga.Box(c["shape"], c["lengths"], chem, diff, c["dt"]) for _ in range(2)]
    outs = [tuple(pinned(np.zeros_like(a)) for a in src) for _ in range(2)]
    for j in range(4):
        b, prev = boxes[j % 2], boxes[(j + 1) % 2]
        b.upload_async(*src)
        if j > 0:
            prev.sync()
            prev.download_async(*outs[(j - 1) % 2])
        b.step(1, graph=True)
    boxes[1].sync()
    boxes[1].download_async(*outs[1])
    for b in boxes:
        b.sync()
    for o in outs:
        for got, exp in zip(o, want):
            assert np.array_equal(got, exp)
