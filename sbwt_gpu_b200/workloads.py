"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is named by the reference or the benchmark definitions, so
every genome, read set and query mix is generated here from a seed (numpy
PCG64), with the shapes, sizes and value distributions of each configuration:

1. small:      uniform-ACGT 1,000,000 bp genome, k=31, p=10; 10,000 reads of 150 bp,
               50% genome-sampled with 1% substitutions, 50% uniform random.
2. large:      100 Mbp genome at 41% GC plus 5% of its length as inserted copies of
               1-10 kbp segments mutated at 0.1%; k=31, p=12; 10M reads of 150 bp,
               10% genome-sampled with 1% substitutions, 90% uniform random.
3. batched:    index of 1; 64 query files with a read-length mixture (70% 150 bp,
               20% lognormal median 2 kbp sigma 1.0, 10% lognormal median 15 kbp
               sigma 0.8, clipped to [31, 100000]); 30% of reads genome-sampled
               with 2% substitutions.
4. prefilter:  index of 1; k-mer queries with 90% negatives (half uniform random,
               half indexed k-mers with 1-3 substitutions).
5. pangenome:  20 haplotypes of a 50 Mbp base (41% GC) with 0.5% SNPs and 0.05%
               indels of 1-20 bp.
``scale`` shrinks a configuration proportionally for tests.
"""
import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def rng_for(seed):
    return np.random.Generator(np.random.PCG64(seed))


def random_bases(rng, n, gc=0.5):
    """n i.i.d. bases with P(G)=P(C)=gc/2, P(A)=P(T)=(1-gc)/2, as ASCII."""
    if gc == 0.5:
        return ACGT[rng.integers(0, 4, size=n, dtype=np.uint8)]
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return ACGT[rng.choice(4, size=n, p=p).astype(np.uint8)]


def substitute(rng, seqs, rate):
    """Each base replaced, with probability `rate`, by one of the 3 other bases (in place)."""
    flat = seqs.reshape(-1)
    hit = np.flatnonzero(rng.random(flat.size) < rate)
    if hit.size:
        codes = np.searchsorted(ACGT, flat[hit])
        flat[hit] = ACGT[(codes + rng.integers(1, 4, size=hit.size)) % 4]
    return seqs


def with_repeats(rng, genome, total, lo=1000, hi=10000, mut=0.001):
    """Inserts copies of random segments (length U[lo, hi]) until `total` bases were added."""
    pieces, cuts, added = [], [], 0
    while added < total:
        ln = int(min(rng.integers(lo, hi + 1), total - added))
        src = int(rng.integers(0, genome.size - ln))
        seg = genome[src:src + ln].copy()
        substitute(rng, seg, mut)
        pieces.append(seg)
        cuts.append(int(rng.integers(0, genome.size)))
        added += ln
    order = np.argsort(cuts, kind="stable")
    out, prev = [], 0
    for i in order:
        out.append(genome[prev:cuts[i]])
        out.append(pieces[i])
        prev = cuts[i]
    out.append(genome[prev:])
    return np.concatenate(out)


def sampled_reads(rng, genome, n, length, sub_rate):
    starts = rng.integers(0, genome.size - length + 1, size=n)
    idx = starts[:, None] + np.arange(length)[None, :]
    reads = genome[idx]
    return substitute(rng, reads, sub_rate)


def uniform_reads(rng, n, length):
    return ACGT[rng.integers(0, 4, size=(n, length), dtype=np.uint8)]


def mixed_reads(rng, genome, n_pos, n_neg, length, sub_rate):
    """n_pos genome-sampled + n_neg random reads of one length, shuffled: (letters, row_starts)."""
    reads = np.concatenate([sampled_reads(rng, genome, n_pos, length, sub_rate), uniform_reads(rng, n_neg, length)])
    reads = reads[rng.permutation(reads.shape[0])]
    rows = np.arange(reads.shape[0] + 1, dtype=np.uint64) * np.uint64(length)
    return np.ascontiguousarray(reads).reshape(-1), rows


def small_workload(seed=1235, scale=1.0):
    rng = rng_for(seed)
    genome = random_bases(rng, int(1_000_000 * scale))
    n_reads = max(2, int(10_000 * scale))
    letters, rows = mixed_reads(rng, genome, n_reads // 2, n_reads - n_reads // 2, 150, 0.01)
    return {"name": "small", "genome": genome, "letters": letters, "row_starts": rows, "k": 31, "p": 10}


def large_workload(seed=1236, scale=1.0, reads_scale=None):
    rng = rng_for(seed)
    n = int(100_000_000 * scale)
    genome = random_bases(rng, n, gc=0.41)
    genome = with_repeats(rng, genome, int(0.05 * n))
    rs = scale if reads_scale is None else reads_scale
    n_reads = max(10, int(10_000_000 * rs))
    n_pos = n_reads // 10
    letters, rows = mixed_reads(rng, genome, n_pos, n_reads - n_pos, 150, 0.01)
    return {"name": "large", "genome": genome, "letters": letters, "row_starts": rows, "k": 31, "p": 12}


def read_lengths(rng, n):
    """70% 150 bp, 20% lognormal(median 2 kbp, sigma 1.0), 10% lognormal(median 15 kbp, sigma 0.8), in [31, 1e5]."""
    u = rng.random(n)
    ln = np.full(n, 150, dtype=np.int64)
    m1 = (u >= 0.7) & (u < 0.9)
    m2 = u >= 0.9
    ln[m1] = np.exp(np.log(2000) + 1.0 * rng.standard_normal(int(m1.sum())))
    ln[m2] = np.exp(np.log(15000) + 0.8 * rng.standard_normal(int(m2.sum())))
    return np.clip(ln, 31, 100_000)


def uneven_read_files(genome, seed=1237, total_kmers=500_000_000, n_files=64, k=31, pos_frac=0.3, sub=0.02):
    """Yields (letters, row_starts) for each of n_files query files until total_kmers k-mers."""
    rng = rng_for(seed)
    per_file = total_kmers // n_files
    for f in range(n_files):
        want = per_file if f < n_files - 1 else total_kmers - per_file * (n_files - 1)
        lens = []
        got = 0
        while got < want:
            ln = read_lengths(rng, 1024)
            for x in ln.tolist():
                lens.append(x)
                got += x - k + 1
                if got >= want:
                    break
        lens = np.array(lens, dtype=np.int64)
        lens[-1] -= got - want  # exact k-mer count
        rows = np.zeros(lens.size + 1, dtype=np.uint64)
        rows[1:] = np.cumsum(lens)
        letters = np.empty(int(rows[-1]), dtype=np.uint8)
        pos = rng.random(lens.size) < pos_frac
        for i, (ln, p) in enumerate(zip(lens.tolist(), pos.tolist())):
            a, b = int(rows[i]), int(rows[i + 1])
            if p and ln <= genome.size:
                s = int(rng.integers(0, genome.size - ln + 1))
                seg = genome[s:s + ln].copy()
                substitute(rng, seg, sub)
                letters[a:b] = seg
            else:
                letters[a:b] = ACGT[rng.integers(0, 4, size=ln, dtype=np.uint8)]
        yield letters, rows


def kmer_queries(rng, genome, n, k, neg_frac=0.9):
    """n single k-mers as rows of length k: (1-neg_frac) indexed, neg_frac/2 random, neg_frac/2 mutated (1-3 subs)."""
    n_neg = int(n * neg_frac)
    n_pos = n - n_neg
    n_rand = n_neg // 2
    n_mut = n_neg - n_rand
    pos = sampled_reads(rng, genome, n_pos, k, 0.0)
    rnd = uniform_reads(rng, n_rand, k)
    mut = sampled_reads(rng, genome, n_mut, k, 0.0)
    nsub = rng.integers(1, 4, size=n_mut)
    for j in range(3):
        rows = np.flatnonzero(nsub > j)
        col = rng.integers(0, k, size=rows.size)
        codes = np.searchsorted(ACGT, mut[rows, col])
        mut[rows, col] = ACGT[(codes + rng.integers(1, 4, size=rows.size)) % 4]
    q = np.concatenate([pos, rnd, mut])
    q = q[rng.permutation(q.shape[0])]
    rows = np.arange(q.shape[0] + 1, dtype=np.uint64) * np.uint64(k)
    return np.ascontiguousarray(q).reshape(-1), rows


def haplotypes(rng, base, n, snp=0.005, indel=0.0005, indel_max=20):
    out = []
    for _ in range(n):
        h = base.copy()
        substitute(rng, h, snp)
        n_ind = rng.binomial(h.size, indel)
        at = np.sort(rng.integers(0, h.size, size=n_ind))
        ln = rng.integers(1, indel_max + 1, size=n_ind)
        ins = rng.random(n_ind) < 0.5
        parts, prev = [], 0
        for a, l, is_ins in zip(at.tolist(), ln.tolist(), ins.tolist()):
            if a < prev:
                continue
            parts.append(h[prev:a])
            if is_ins:
                parts.append(ACGT[rng.integers(0, 4, size=l, dtype=np.uint8)])
                prev = a
            else:
                prev = min(a + l, h.size)
        parts.append(h[prev:])
        out.append(np.concatenate(parts))
    return out


def write_fastq(path, letters, row_starts, crlf=False):
    """Writes rows as FASTQ records (@header, sequence, '+', qualities of the same length)."""
    rs = np.asarray(row_starts, dtype=np.int64)
    eol = b"\r\n" if crlf else b"\n"
    with open(path, "wb") as f:
        for i in range(rs.size - 1):
            seq = letters[rs[i]:rs[i + 1]].tobytes()
            f.write(b"@r%d length=%d" % (i, len(seq)) + eol + seq + eol + b"+" + eol + b"I" * len(seq) + eol)


def write_fasta(path, letters, row_starts, width=None):
    """Writes rows as FASTA records (one header + one sequence line each, '\\n'-terminated)."""
    rs = np.asarray(row_starts, dtype=np.int64)
    with open(path, "wb") as f:
        for i in range(rs.size - 1):
            f.write(b">r%d\n" % i)
            f.write(letters[rs[i]:rs[i + 1]].tobytes())
            f.write(b"\n")


def pack_words(seq):
    """ASCII ACGT -> MSB-first 2-bit words (letter i of word w at bits 63-2i..62-2i), plus one zero word."""
    codes = np.searchsorted(ACGT, seq).astype(np.uint64)
    n = codes.size
    nw = (n + 31) // 32 + 1
    padded = np.zeros(nw * 32, dtype=np.uint64)
    padded[:n] = codes
    p = padded.reshape(nw, 32)
    words = np.zeros(nw, dtype=np.uint64)
    for i in range(32):
        words |= p[:, i] << np.uint64(62 - 2 * i)
    return words


def kmer_query_words(rng, genome, n, k, neg_frac=0.9, chunk=10_000_000):
    """n k-mers as MSB-first u64 words: (1-neg_frac) sampled from the genome, neg_frac/2 uniform random,
    neg_frac/2 genome k-mers with 1-3 substitutions; shuffled."""
    words = pack_words(genome)
    mask = np.uint64(((1 << (2 * k)) - 1) << (64 - 2 * k)) if k < 32 else np.uint64(0xFFFFFFFFFFFFFFFF)
    out = np.empty(n, dtype=np.uint64)
    n_neg = int(n * neg_frac)
    kinds = np.zeros(n, dtype=np.uint8)  # 0 genome, 1 random, 2 mutated
    kinds[: n_neg // 2] = 1
    kinds[n_neg // 2: n_neg] = 2
    rng.shuffle(kinds)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        kd = kinds[a:b]
        pos = rng.integers(0, genome.size - k + 1, size=b - a).astype(np.uint64)
        wi = (pos >> np.uint64(5)).astype(np.int64)
        sh = (pos & np.uint64(31)) * np.uint64(2)
        hi = words[wi] << sh
        lo = np.where(sh == 0, np.uint64(0), words[wi + 1] >> (np.uint64(64) - np.where(sh == 0, np.uint64(1), sh)))
        x = (hi | lo) & mask
        mut = kd == 2
        nsub = rng.integers(1, 4, size=b - a)
        for s in range(3):
            sel = mut & (nsub > s)
            p = rng.integers(0, k, size=b - a).astype(np.uint64)
            shift = np.uint64(62) - np.uint64(2) * p
            old = (x >> shift) & np.uint64(3)
            new = (old + rng.integers(1, 4, size=b - a).astype(np.uint64)) & np.uint64(3)
            x = np.where(sel, (x & ~(np.uint64(3) << shift)) | (new << shift), x)
        rnd = rng.integers(0, 2**63, size=b - a, dtype=np.int64).astype(np.uint64) * np.uint64(2) & mask
        out[a:b] = np.where(kd == 1, rnd, x)
    return out
