"""sbwt_search_reads_noalloc: the search for callers that cannot call
cudaMalloc while they search (a process whose device memory another allocator
already holds, or an application that accounts for every device allocation
itself).  Its scratch is a fixed device array inside the library instead of
buffers grown with cudaMalloc.

Checked through the C ABI against sbwt_search_reads and the oracle on the same batch, on two
calls in a row (the array keeps the previous call's contents, so the second
call shows that nothing stale leaks into its answers), in the default run walk
and with every k-mer searched, on the line and the poppy layouts, with answers
and bitmap and with the bitmap alone; a batch beyond the array's size is
rejected with an error.  Answers are integers: they must be equal.  This file
is collected last so that a failure here leaves every other test already run.
"""
from ctypes import c_void_p

import numpy as np
import pytest

import oracle as orc
import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import _lib, workloads as wl

pytestmark = pytest.mark.gpu


def _noalloc(ix, d_letters, d_rows, d_answers, n_kmers, d_member=None, stream=None):
    return _lib.lib.sbwt_search_reads_noalloc(ix._h, c_void_p(d_letters.data_ptr()), d_letters.numel(),
                                              c_void_p(d_rows.data_ptr()), d_rows.numel() - 1,
                                              c_void_p(d_answers.data_ptr()) if d_answers is not None else None,
                                              c_void_p(d_member.data_ptr()) if d_member is not None else None,
                                              n_kmers, None)


@pytest.mark.parametrize("layout", ["lines", "poppy"])
@pytest.mark.parametrize("mode", ["stream", "every"])
def test_noalloc_search_equals_search_reads(cuda, layout, mode):
    import torch
    rng = wl.rng_for(606)
    genome = wl.random_bases(rng, 200_000)
    built = sg.build_sbwt([genome.tobytes()], 31)
    batches = [wl.mixed_reads(rng, genome, 400, 400, 150, 0.01),
               wl.mixed_reads(rng, genome, 50, 150, 90, 0.02)]  # second call: a smaller, different batch
    kw = dict(k=31, k_presearch=10, search_mode=sg.SEARCH_STREAM if mode == "stream" else sg.SEARCH_EVERY_KMER)
    if layout == "poppy":
        kw.update(layout=sg.SBWT_LAYOUT_POPPY, bits_in_superblock=1024)
    ox = orc.OracleIndex(built.bits, built.n_bits)
    with sg.Index.from_bits(built.bits, built.n_bits, **kw) as ix:
        for letters, rows in batches:
            nk = sg.count_kmers(rows, 31)
            d_l = torch.from_numpy(letters).to(cuda)
            d_r = torch.from_numpy(rows.view(np.int64)).to(cuda)
            want = torch.empty(nk, dtype=torch.int64, device=cuda)
            want_bits = torch.zeros((nk + 31) // 32, dtype=torch.int32, device=cuda)
            ix.search_reads(d_l, d_r, want, nk, d_member_bits=want_bits)
            got = torch.full((nk,), -3, dtype=torch.int64, device=cuda)
            got_bits = torch.full(((nk + 31) // 32,), -1, dtype=torch.int32, device=cuda)
            assert _noalloc(ix, d_l, d_r, got, nk, got_bits) == 0, _lib.lib.sbwt_last_error()
            torch.cuda.synchronize()
            assert torch.equal(got, want)
            assert torch.equal(got_bits, want_bits)
            # and against the oracle itself, so that a fault shared with sbwt_search_reads shows too
            assert np.array_equal(got.cpu().numpy().view(np.uint64), ox.search_reads(letters, rows, 31, 10))
            # membership only: no answer array
            only_bits = torch.full(((nk + 31) // 32,), -1, dtype=torch.int32, device=cuda)
            assert _noalloc(ix, d_l, d_r, None, nk, only_bits) == 0, _lib.lib.sbwt_last_error()
            torch.cuda.synchronize()
            assert torch.equal(only_bits, want_bits)


def test_noalloc_rejects_a_batch_beyond_its_scratch(cuda):
    import torch
    rng = wl.rng_for(607)
    genome = wl.random_bases(rng, 50_000)
    built = sg.build_sbwt([genome.tobytes()], 31)
    with sg.Index.from_bits(built.bits, built.n_bits, k=31, k_presearch=8) as ix:
        n_letters = 160 << 20  # 160M letters: their packed words alone exceed the 32 MiB scratch
        d_l = torch.full((n_letters,), ord("A"), dtype=torch.uint8, device=cuda)
        d_r = torch.tensor([0, n_letters], dtype=torch.int64, device=cuda)
        d_a = torch.empty(1, dtype=torch.int64, device=cuda)
        assert _noalloc(ix, d_l, d_r, d_a, n_letters - 30) != 0
        err = _lib.lib.sbwt_last_error()
        assert b"scratch" in err and b"bytes" in err
        assert _noalloc(ix, d_l, d_r, None, n_letters - 30) != 0  # NULL answers and no bitmap
        assert b"NULL" in _lib.lib.sbwt_last_error()
