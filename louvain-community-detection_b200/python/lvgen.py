"""Seeded synthetic graphs with the shapes of the benchmark workloads, and
Matrix Market I/O with the reference reader's semantics.

Every generator returns an undirected edge list (src, dst, w) in "file
order"; `csr_from_edges` turns it into the CSR the reference's reader
builds from the same lines (utils.cu:200-227: each edge stored in both
rows, a self-loop once, every row in file order).

Workloads (sizes as in the benchmark descriptions):
  banded_fem      symmetric banded FEM-like matrix (n=4,884, half-band 60,
                  ~290k stored entries, weights U(0.1, 1.0))
  planted_powerlaw  Chung-Lu degrees (exponent 2.3, max 550) with planted
                  LFR-style communities (size exponent 1.5, mixing mu)
  rmat            R-MAT (a, b, c, d) = (.57, .19, .19, .05), duplicates
                  merged, self-loops dropped
  sbm             stochastic block model with p_in / p_out = 20
"""
from __future__ import annotations

import numpy as np

F32 = np.float32


def csr_from_edges(n: int, src: np.ndarray, dst: np.ndarray,
                   w: np.ndarray):
    """CSR (off u64[n+1], col u32[E], w f32[E]) with the reference layout."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    w = np.asarray(w, dtype=F32)
    m = len(src)
    loop = src == dst
    # entries in file order: edge i contributes (src->dst) then (dst->src)
    rows = np.empty(2 * m, dtype=np.int64)
    cols = np.empty(2 * m, dtype=np.int64)
    ws = np.empty(2 * m, dtype=F32)
    rows[0::2], rows[1::2] = src, dst
    cols[0::2], cols[1::2] = dst, src
    ws[0::2], ws[1::2] = w, w
    keep = np.ones(2 * m, dtype=bool)
    keep[1::2] = ~loop
    rows, cols, ws = rows[keep], cols[keep], ws[keep]
    order = np.argsort(rows, kind="stable")
    rows, cols, ws = rows[order], cols[order], ws[order]
    deg = np.bincount(rows, minlength=n).astype(np.uint64)
    off = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(deg, out=off[1:])
    return off, cols.astype(np.uint32), ws


def write_mtx(path: str, n: int, src, dst, w, one_based: bool = True,
              banner: bool = False, comments=(), with_weights: bool = True):
    """Writes `rows cols nnz` + `i j w` lines (readable by both the
    reference CLI and louvian.py when banner/comments are off)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    w = np.asarray(w, dtype=F32)
    b = 1 if one_based else 0
    with open(path, "w") as f:
        if banner:
            f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        for c in comments:
            f.write("%" + c + "\n")
        f.write(f"{n} {n} {len(src)}\n")
        if with_weights:
            # The shortest repr of the float32 value taken as a double parses
            # to that same value with strtof (reference CLI) and with float()
            # (louvian.py), so both readers see identical weights.
            for a, c, x in zip(src.tolist(), dst.tolist(), _fmt_weights(w)):
                f.write(f"{a + b} {c + b} {x}\n")
        else:
            for a, c in zip(src.tolist(), dst.tolist()):
                f.write(f"{a + b} {c + b}\n")


def _fmt_weights(w):
    return [repr(float(np.float32(x))) for x in w]


def banded_fem(n: int = 4884, half_band: int = 60, target_entries: int = 290_000,
               seed: int = 0):
    """Lower-triangle banded matrix (diagonal included), listed column by
    column like a Harwell-Boeing stiffness matrix."""
    rng = np.random.default_rng(seed)
    # off-diagonal pairs needed so that 2*offdiag + n ~= target_entries
    off_pairs = max(0, (target_entries - n) // 2)
    full = sum(min(half_band, n - 1 - j) for j in range(n))
    p = min(1.0, off_pairs / max(full, 1))
    src, dst = [], []
    for j in range(n):
        src.append(j)
        dst.append(j)
        hi = min(n - 1, j + half_band)
        if hi > j:
            rows = np.arange(j + 1, hi + 1)
            rows = rows[rng.random(len(rows)) < p]
            src.extend(rows.tolist())
            dst.extend([j] * len(rows))
    src = np.array(src, dtype=np.int64)
    dst = np.array(dst, dtype=np.int64)
    w = rng.uniform(0.1, 1.0, size=len(src)).astype(F32)
    return n, src, dst, w


def _powerlaw_ints(rng, size, exponent, lo, hi):
    """Discrete power law P(k) ~ k^-exponent on [lo, hi]."""
    ks = np.arange(lo, hi + 1, dtype=np.float64)
    p = ks ** (-exponent)
    p /= p.sum()
    return rng.choice(np.arange(lo, hi + 1), size=size, p=p)


def planted_powerlaw(n: int = 334_863, target_edges: int = 925_872,
                     gamma: float = 2.3, max_deg: int = 550, mu: float = 0.3,
                     comm_exp: float = 1.5, comm_min: int = 10,
                     comm_max: int = 2000, seed: int = 0, unit: bool = True):
    """Chung-Lu style degrees with planted communities (LFR-like):
    a (1-mu) share of each vertex's stubs pairs inside its community, the
    rest pairs globally; duplicates and self-loops are removed."""
    # Degrees follow a continuous power law on [xmin, max_deg], rounded; the
    # stub budget is calibrated (two deterministic rounds) so that the
    # simple graph left after removing loops and duplicates has about
    # target_edges edges.
    scale = 1.0
    for _ in range(3):
        src, dst, comm_of, sizes = _planted_edges(n, target_edges * scale, gamma,
                                                  max_deg, mu, comm_exp, comm_min,
                                                  comm_max, seed)
        got = len(src)
        if abs(got - target_edges) <= 0.002 * target_edges:
            break
        scale *= target_edges / max(got, 1)
    rng = np.random.default_rng(seed + 7919)
    w = np.ones(len(src), dtype=F32) if unit else \
        rng.uniform(0.5, 1.5, len(src)).astype(F32)
    return n, src, dst, w


def _cont_powerlaw_mean(gamma, xmin, xmax):
    a, b = 1.0 - gamma, 2.0 - gamma
    return (a / b) * (xmax ** b - xmin ** b) / (xmax ** a - xmin ** a)


def _planted_edges(n, target_edges, gamma, max_deg, mu, comm_exp, comm_min,
                   comm_max, seed):
    rng = np.random.default_rng(seed)
    mean_target = 2.0 * target_edges / n
    lo, hi = 0.5, 60.0
    for _ in range(60):  # xmin giving the target mean
        mid = 0.5 * (lo + hi)
        if _cont_powerlaw_mean(gamma, mid, max_deg) < mean_target:
            lo = mid
        else:
            hi = mid
    xmin = 0.5 * (lo + hi)
    a = 1.0 - gamma
    u = rng.random(n)
    x = ((max_deg ** a - xmin ** a) * u + xmin ** a) ** (1.0 / a)
    deg = np.clip(np.rint(x), 1, max_deg).astype(np.int64)
    # community sizes ~ power law (exponent comm_exp) covering n vertices
    sizes = []
    total = 0
    while total < n:
        s = int(_powerlaw_ints(rng, 1, comm_exp, comm_min, comm_max)[0])
        s = min(s, n - total)
        sizes.append(s)
        total += s
    sizes = np.array(sizes, dtype=np.int64)
    perm = rng.permutation(n)
    comm_of = np.empty(n, dtype=np.int64)
    comm_of[perm] = np.repeat(np.arange(len(sizes)), sizes)
    k_in = np.rint((1.0 - mu) * deg).astype(np.int64)
    # a vertex cannot have more intra stubs than its community can absorb
    k_in = np.minimum(k_in, sizes[comm_of] - 1)
    k_out = deg - k_in
    # intra: configuration model inside every community
    stub_v = np.repeat(np.arange(n), k_in)
    key = comm_of[stub_v].astype(np.float64) + rng.random(len(stub_v))
    stub_v = stub_v[np.argsort(key, kind="stable")]
    stub_c = comm_of[stub_v]
    # pair consecutive stubs of the same community
    same = np.zeros(len(stub_v), dtype=bool)
    if len(stub_v) > 1:
        # greedy: take pairs (0,1),(2,3)... within each community run
        starts = np.flatnonzero(np.r_[True, stub_c[1:] != stub_c[:-1]])
        idx = np.arange(len(stub_v))
        run_start = np.repeat(starts, np.diff(np.r_[starts, len(stub_v)]))
        pos = idx - run_start
        first = (pos % 2 == 0) & (idx + 1 < len(stub_v))
        first &= np.r_[stub_c[1:] == stub_c[:-1], False]
        same = first
    a1 = stub_v[same]
    b1 = stub_v[np.flatnonzero(same) + 1]
    # inter: global configuration model
    stub_o = np.repeat(np.arange(n), k_out)
    stub_o = stub_o[rng.permutation(len(stub_o))]
    h = len(stub_o) // 2
    a2, b2 = stub_o[:h], stub_o[h:2 * h]
    src = np.concatenate([a1, a2])
    dst = np.concatenate([b1, b2])
    src, dst = _simple(n, src, dst, rng)
    return src, dst, comm_of, sizes


def _simple(n, src, dst, rng, shuffle=True):
    """Drops self-loops and duplicate undirected edges; random file order."""
    keep = src != dst
    src, dst = src[keep], dst[keep]
    lo = np.minimum(src, dst)
    hi = np.maximum(src, dst)
    key = lo * np.int64(n) + hi
    _, first = np.unique(key, return_index=True)
    src, dst = src[first], dst[first]
    if shuffle:
        p = rng.permutation(len(src))
        src, dst = src[p], dst[p]
    return src, dst


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19,
         seed: int = 0, unit: bool = True):
    """R-MAT edges (duplicates merged, self-loops dropped)."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    m = edge_factor * n
    src = np.zeros(m, dtype=np.int64)
    dst = np.zeros(m, dtype=np.int64)
    ab, abc = a + b, a + b + c
    for lvl in range(scale):
        r = rng.random(m)
        bit = np.int64(1) << (scale - 1 - lvl)
        down = r >= ab  # quadrants c, d: row bit set
        right = ((r >= a) & (r < ab)) | (r >= abc)  # quadrants b, d
        src += np.where(down, bit, 0)
        dst += np.where(right, bit, 0)
    src, dst = _simple(n, src, dst, rng)
    w = np.ones(len(src), dtype=F32) if unit else \
        rng.uniform(0.1, 1.0, len(src)).astype(F32)
    return n, src, dst, w


def rmat_device(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19,
                seed: int = 0, device: str = "cuda"):
    """R-MAT generated and symmetrised on the GPU (torch), for sizes numpy
    cannot produce quickly (scale 24: 268M draws, 537M stored entries).
    Duplicates merged, self-loops dropped, unit weights.  Returns
    (n, off int64[n+1], col int32[E], w float32[E], n_edges) as device
    tensors; a row lists its higher-numbered neighbours, then its
    lower-numbered ones, each group ascending."""
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    n = 1 << scale
    m = edge_factor * n
    src = torch.zeros(m, dtype=torch.int64, device=device)
    dst = torch.zeros(m, dtype=torch.int64, device=device)
    ab, abc = a + b, a + b + c
    for lvl in range(scale):
        r = torch.rand(m, generator=gen, device=device)
        bit = 1 << (scale - 1 - lvl)
        src += (r >= ab).to(torch.int64) * bit
        dst += (((r >= a) & (r < ab)) | (r >= abc)).to(torch.int64) * bit
        del r
    keep = src != dst
    lo = torch.minimum(src, dst)[keep]
    hi = torch.maximum(src, dst)[keep]
    del src, dst, keep
    key = torch.unique(lo * n + hi)  # sorted, duplicates merged
    del lo, hi
    lo = key // n
    hi = key % n
    del key
    n_edges = int(lo.numel())
    rows = torch.cat([lo, hi])
    cols = torch.cat([hi, lo])
    del lo, hi
    rows, order = torch.sort(rows, stable=True)
    cols = cols[order].to(torch.int32)
    del order
    counts = torch.bincount(rows, minlength=n)
    del rows
    off = torch.zeros(n + 1, dtype=torch.int64, device=device)
    off[1:] = torch.cumsum(counts, 0)
    w = torch.ones(cols.numel(), dtype=torch.float32, device=device)
    return n, off, cols, w, n_edges


def sbm_batch_sizes(count: int, seed: int = 0, lo: int = 64, hi: int = 65_536,
                    min_blocks: int = 4, max_blocks: int = 32):
    """Per-graph vertex and block counts of a batch: sizes log-uniform in
    [lo, hi], blocks uniform in [min_blocks, max_blocks] (at most n/4)."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count)).astype(np.int64)
    n = np.clip(n, lo, hi)
    b = rng.integers(min_blocks, max_blocks + 1, count)
    b = np.maximum(1, np.minimum(b, n // 4))
    return n, b


def sbm_batch_device(count: int, seed: int = 0, lo: int = 64, hi: int = 65_536,
                     mean_deg: float = 16.0, ratio: float = 20.0, wlo: float = 0.5,
                     whi: float = 1.5, device: str = "cuda"):
    """`count` stochastic-block-model graphs (sizes from sbm_batch_sizes,
    equal blocks, p_in/p_out = ratio, mean degree mean_deg, weights
    U(wlo, whi)) generated on the device (torch) and packed as one
    block-diagonal union CSR.  Intra-block edges pick a block uniformly and
    two of its members; inter-block edges a vertex and a member of another
    block.  Duplicates merged, self-loops dropped.  Returns (goff u64[G+1]
    numpy, off int64[N+1], col int32[E], w float32[E], n_edges) with the
    tensors on `device`; graph g owns vertices [goff[g], goff[g+1])."""
    import torch

    ns, bs = sbm_batch_sizes(count, seed, lo, hi)
    goff = np.zeros(count + 1, dtype=np.uint64)
    goff[1:] = np.cumsum(ns)
    N = int(goff[-1])
    # expected edge counts per graph
    s = ns / bs
    p_out = mean_deg / (ratio * (s - 1) + (ns - s))
    p_in = ratio * p_out
    m_in = np.rint(p_in * bs * s * (s - 1) / 2).astype(np.int64)
    m_out = np.rint(p_out * (ns * (ns - 1) / 2 - bs * s * (s - 1) / 2)).astype(np.int64)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    t_n, t_b = T(ns), T(bs)
    t_base = T(goff[:-1].astype(np.int64))

    def member(g, blk):
        # vertex of block blk of graph g; blocks of size n//B, the first
        # n % B of them one larger
        q, r = t_n[g] // t_b[g], t_n[g] % t_b[g]
        start = blk * q + torch.minimum(blk, r)
        size = q + (blk < r).to(torch.int64)
        off = (torch.rand(g.numel(), generator=gen, device=device) * size).to(torch.int64)
        return t_base[g] + start + torch.minimum(off, size - 1)

    gi = torch.repeat_interleave(torch.arange(count, device=device), T(m_in))
    blk = (torch.rand(gi.numel(), generator=gen, device=device) * t_b[gi]).to(torch.int64)
    blk = torch.minimum(blk, t_b[gi] - 1)
    u1, v1 = member(gi, blk), member(gi, blk)
    go = torch.repeat_interleave(torch.arange(count, device=device), T(m_out))
    bo = torch.minimum((torch.rand(go.numel(), generator=gen, device=device) * t_b[go])
                       .to(torch.int64), t_b[go] - 1)
    shift = 1 + torch.minimum((torch.rand(go.numel(), generator=gen, device=device)
                               * (t_b[go] - 1)).to(torch.int64),
                              torch.clamp(t_b[go] - 2, min=0))
    keep_o = t_b[go] > 1
    u2 = member(go, bo)
    v2 = member(go, (bo + shift) % t_b[go])
    u2, v2 = u2[keep_o], v2[keep_o]
    src = torch.cat([u1, u2])
    dst = torch.cat([v1, v2])
    del u1, v1, u2, v2, gi, blk, go, bo, shift
    keep = src != dst
    lo_ = torch.minimum(src, dst)[keep]
    hi_ = torch.maximum(src, dst)[keep]
    del src, dst, keep
    key = torch.unique(lo_ * N + hi_)
    del lo_, hi_
    a, b = key // N, key % N
    del key
    n_edges = int(a.numel())
    w1 = torch.rand(n_edges, generator=gen, device=device) * (whi - wlo) + wlo
    rows = torch.cat([a, b])
    cols = torch.cat([b, a])
    ww = torch.cat([w1, w1]).to(torch.float32)
    del a, b, w1
    rows, order = torch.sort(rows, stable=True)
    cols = cols[order].to(torch.int32)
    ww = ww[order]
    del order
    counts = torch.bincount(rows, minlength=N)
    del rows
    off = torch.zeros(N + 1, dtype=torch.int64, device=device)
    off[1:] = torch.cumsum(counts, 0)
    return goff, off, cols, ww, n_edges


def _csr_device(n, a, b, device):
    """Symmetric CSR (rows ascending, each row's entries in key order) of
    the undirected edges a < b (int64 tensors), unit FP32 weights."""
    import torch

    rows = torch.cat([a, b])
    cols = torch.cat([b, a])
    rows, order = torch.sort(rows, stable=True)
    cols = cols[order].to(torch.int32)
    del order
    counts = torch.bincount(rows, minlength=n)
    del rows
    off = torch.zeros(n + 1, dtype=torch.int64, device=device)
    off[1:] = torch.cumsum(counts, 0)
    w = torch.ones(cols.numel(), dtype=torch.float32, device=device)
    return off, cols, w


def lfr_device(n: int, mu: float, seed: int = 0, gamma: float = 2.3, beta: float = 1.5,
               mean_deg: float = 16.0, cmin: int = 20, device: str = "cuda"):
    """LFR-style benchmark graph generated on the device (torch): vertex
    degrees from a power law (exponent gamma, mean about mean_deg, maximum
    about 2 sqrt(n)), community sizes from a power law (exponent beta,
    cmin .. n/10), a fraction mu of every vertex's edges to uniform random
    vertices and the rest to uniform members of its own community (the
    degree cap and merged duplicates leave a mean degree somewhat below
    mean_deg).  Self-loops dropped, unit FP32 weights.  Returns
    (n, off int64[n+1], col int32[E], w float32[E], n_edges) on `device`
    and the community of every vertex (numpy)."""
    import torch

    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    # community sizes, then a random placement of vertices into them
    cmax = max(cmin + 1, n // 10)
    sizes = []
    total = 0
    while total < n:
        u = rng.random()
        lo_, hi_ = cmin ** (1 - beta), cmax ** (1 - beta)
        s = int((lo_ + u * (hi_ - lo_)) ** (1 / (1 - beta)))
        s = min(max(s, cmin), n - total) if n - total >= cmin else n - total
        sizes.append(s)
        total += s
    sizes = np.array(sizes, dtype=np.int64)
    starts = np.r_[0, np.cumsum(sizes)[:-1]]
    perm = rng.permutation(n)  # position p of the community layout -> vertex id
    comm_of_pos = np.repeat(np.arange(len(sizes)), sizes)
    comm = np.empty(n, dtype=np.int64)
    comm[perm] = comm_of_pos
    # degrees (halved: every stub makes one edge, seen from both ends)
    kmax = max(8.0, 2.0 * np.sqrt(n))
    kmin = max(1.0, mean_deg * (gamma - 2) / (gamma - 1))
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(device)
    u = torch.rand(n, generator=gen, device=device, dtype=torch.float64)
    deg = kmin * (1 - u) ** (-1.0 / (gamma - 1))
    deg = torch.clamp(deg, max=kmax)
    stubs = torch.clamp((deg / 2).round().to(torch.int64), min=1)
    pos_of_v = T(np.argsort(perm))  # vertex -> layout position
    t_perm, t_sizes, t_starts = T(perm), T(sizes), T(starts)
    t_comm = T(comm)
    src = torch.repeat_interleave(torch.arange(n, device=device), stubs)
    m = src.numel()
    ext = torch.rand(m, generator=gen, device=device) < mu
    c = t_comm[src]
    r = torch.rand(m, generator=gen, device=device, dtype=torch.float64)
    internal = t_perm[t_starts[c] + torch.minimum((r * t_sizes[c]).to(torch.int64), t_sizes[c] - 1)]
    external = torch.minimum((r * n).to(torch.int64), torch.tensor(n - 1, device=device))
    dst = torch.where(ext, external, internal)
    del ext, c, r, internal, external, pos_of_v
    keep = src != dst
    a = torch.minimum(src, dst)[keep]
    b = torch.maximum(src, dst)[keep]
    del src, dst, keep
    key = torch.unique(a * n + b)
    a, b = key // n, key % n
    del key
    n_edges = int(a.numel())
    off, col, w = _csr_device(n, a, b, device)
    return (n, off, col, w, n_edges), comm


def localize_batch(goff, off, col):
    """Per-graph CSR views of a block-diagonal union, for running the
    graphs one by one: returns (loff int64[N+G], lcol int32[E]) where graph
    g's offsets (n_g+1 of them, starting at 0) sit at loff[goff[g]+g:] and
    its column ids are local (col - goff[g])."""
    import torch

    G = len(goff) - 1
    dev = off.device
    ns = torch.from_numpy((goff[1:] - goff[:-1]).astype(np.int64)).to(dev)
    gid_v = torch.repeat_interleave(torch.arange(G, device=dev), ns)
    base_v = torch.from_numpy(goff[:-1].astype(np.int64)).to(dev)
    N = int(goff[-1])
    # graph of every entry: gid of its row
    deg = off[1:] - off[:-1]
    gid_e = torch.repeat_interleave(gid_v, deg)
    lcol = (col.to(torch.int64) - base_v[gid_e]).to(torch.int32)
    del gid_e
    e0 = off[base_v]  # first entry of each graph
    loff = torch.empty(N + G, dtype=torch.int64, device=dev)
    pos = torch.arange(N, device=dev) + gid_v  # row v of graph g at goff[g] + g + local
    loff[pos] = off[:-1] - e0[gid_v]
    ends = torch.from_numpy((goff[1:] + np.arange(G, dtype=np.uint64)).astype(np.int64)).to(dev)
    ends_val = off[torch.from_numpy(goff[1:].astype(np.int64)).to(dev)] - e0
    loff[ends] = ends_val
    return loff, lcol


def sbm(n: int, blocks: int, mean_deg: float = 16.0, ratio: float = 20.0,
        seed: int = 0, wlo: float = 0.5, whi: float = 1.5):
    """Stochastic block model with equal blocks, p_in/p_out = ratio, mean
    degree mean_deg, weights U(wlo, whi)."""
    rng = np.random.default_rng(seed)
    bs = n // blocks
    sizes = np.full(blocks, bs, dtype=np.int64)
    sizes[: n - bs * blocks] += 1
    block_of = np.repeat(np.arange(blocks), sizes)
    # expected degree = p_in*(s-1) + p_out*(n-s) = mean_deg
    s = n / blocks
    p_out = mean_deg / (ratio * (s - 1) + (n - s))
    p_in = ratio * p_out
    m_in = int(round(p_in * sum(int(x) * (int(x) - 1) // 2 for x in sizes)))
    m_out = int(round(p_out * (n * (n - 1) // 2 - sum(int(x) * (int(x) - 1) // 2
                                                      for x in sizes))))
    starts = np.r_[0, np.cumsum(sizes)[:-1]]
    # intra edges: pick a block proportional to its pair count, then two members
    pairs = sizes * (sizes - 1) / 2.0
    bsel = rng.choice(blocks, size=m_in, p=pairs / pairs.sum())
    u = starts[bsel] + (rng.random(m_in) * sizes[bsel]).astype(np.int64)
    v = starts[bsel] + (rng.random(m_in) * sizes[bsel]).astype(np.int64)
    # inter edges: two uniform vertices in different blocks
    x = rng.integers(0, n, size=2 * m_out + 16)
    y = rng.integers(0, n, size=2 * m_out + 16)
    ok = block_of[x] != block_of[y]
    x, y = x[ok][:m_out], y[ok][:m_out]
    src = np.concatenate([u, x])
    dst = np.concatenate([v, y])
    src, dst = _simple(n, src, dst, rng)
    w = rng.uniform(wlo, whi, len(src)).astype(F32)
    return n, src, dst, w


def two_cliques_bridge(k: int = 5):
    """Two k-cliques joined by one bridge edge."""
    src, dst = [], []
    for base in (0, k):
        for i in range(k):
            for j in range(i + 1, k):
                src.append(base + i)
                dst.append(base + j)
    src.append(k - 1)
    dst.append(k)
    return 2 * k, np.array(src), np.array(dst), np.ones(len(src), dtype=F32)


def ring_of_cliques(cliques: int = 8, k: int = 6):
    src, dst = [], []
    for c in range(cliques):
        base = c * k
        for i in range(k):
            for j in range(i + 1, k):
                src.append(base + i)
                dst.append(base + j)
        src.append(base + k - 1)
        dst.append(((c + 1) % cliques) * k)
    n = cliques * k
    return n, np.array(src), np.array(dst), np.ones(len(src), dtype=F32)


def star(leaves: int = 1000, seed: int = 0):
    rng = np.random.default_rng(seed)
    src = np.zeros(leaves, dtype=np.int64)
    dst = np.arange(1, leaves + 1)
    w = rng.uniform(0.5, 1.5, leaves).astype(F32)
    return leaves + 1, src, dst, w
