"""The answer text formatted on the GPU against the host formatter and the oracle (needs a B200)."""
import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg

pytestmark = pytest.mark.gpu


def _dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(dev)


@pytest.mark.parametrize("k", [3, 31])
def test_device_text_equals_host_text(cuda, k):
    rng = np.random.default_rng(7 + k)
    lens = rng.integers(0, 200, size=3000)
    lens[:5] = [0, k - 1, k, 0, 0]  # empty rows and rows without k-mers, also at the start
    lens[-3:] = [0, k - 1, 0]      # ... and at the end
    rows = np.zeros(lens.size + 1, dtype=np.uint64)
    rows[1:] = np.cumsum(lens)
    nk = int(np.maximum(lens - k + 1, 0).sum())
    ans = rng.integers(0, 2**40, size=nk, dtype=np.uint64)
    ans[rng.random(nk) < 0.5] = orc.NOT_FOUND
    ans[:3] = [0, 9, 10]
    ans[-3:] = [np.uint64(2**63 - 1), np.uint64(2**63), np.uint64(10**19)]  # the int64 range edges
    want = sg.format_answers(rows, k, ans)
    assert want == orc.format_answers(rows, k, ans)
    got = sg.format_answers_device(_dev(rows, cuda), k, _dev(ans, cuda))
    assert got == want


def test_device_text_without_kmers(cuda):
    rows = np.array([0, 2, 2, 5], dtype=np.uint64)
    got = sg.format_answers_device(_dev(rows, cuda), 31, _dev(np.zeros(0, np.uint64), cuda))
    assert got == b"\n\n\n"


def test_device_text_rejects_a_wrong_kmer_count(cuda):
    rows = np.array([0, 40], dtype=np.uint64)
    with pytest.raises(sg.SbwtError, match="k-mers"):
        sg.format_answers_device(_dev(rows, cuda), 31, _dev(np.zeros(3, np.uint64), cuda))
