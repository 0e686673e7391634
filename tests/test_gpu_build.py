"""The GPU SBWT builder against the host builder, bit for bit (needs a B200)."""
import numpy as np
import pytest

import sbwt_gpu_b200 as sg
from sbwt_gpu_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _same(seqs, k):
    host = sg.build_sbwt(seqs, k)
    gpu = sg.build_sbwt(seqs, k, device=0)
    assert (gpu.n_bits, gpu.n_kmers, gpu.n_dummies) == (host.n_bits, host.n_kmers, host.n_dummies)
    nw = (host.n_bits + 63) // 64
    for c in range(4):
        assert np.array_equal(gpu.bits[c][:nw], host.bits[c][:nw]), c
    return gpu


@pytest.mark.parametrize("k", [3, 4, 7, 12, 31, 32])
@pytest.mark.parametrize("seed", [1, 2])
def test_small_random_sets(cuda, k, seed):
    rng = np.random.default_rng(seed * 1000 + k)
    seqs = ["".join(rng.choice(list("ACGTN"), p=[0.24, 0.24, 0.24, 0.24, 0.04], size=int(rng.integers(1, 400))))
            for _ in range(int(rng.integers(1, 40)))]
    seqs.append("ACGT" * 20)
    _same(seqs, k)


def test_cyclic_set_has_root_only_dummy(cuda):
    g = _same(["ACGTTGCA" * 4], 4)
    assert g.n_dummies == 1


def test_genome_with_repeats(cuda):
    rng = wl.rng_for(5)
    g = wl.random_bases(rng, 300_000, gc=0.41)
    g = wl.with_repeats(rng, g, 20_000)
    _same([g.tobytes()], 31)


def test_haplotypes_and_reads(cuda):
    rng = wl.rng_for(51)
    base = wl.random_bases(rng, 200_000, gc=0.41)
    haps = wl.haplotypes(rng, base, 6)
    _same([h.tobytes() for h in haps], 31)
    # a read set: thousands of short sequences, some shorter than k, lowercase and N
    reads = wl.sampled_reads(rng, base, 3000, 100, 0.01)
    seqs = [r.tobytes() for r in reads] + [b"acgtnnacgt" * 5, b"ACG", b""]
    _same(seqs, 31)


def test_no_kmer_is_an_error(cuda):
    with pytest.raises(sg.SbwtError, match="no k-mer"):
        sg.build_sbwt(["ACG", "NNNNNNNN"], 5, device=0)
