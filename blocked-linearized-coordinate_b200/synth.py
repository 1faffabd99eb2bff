"""Seeded synthetic sparse tensors of the benchmark shapes.

The reference is benchmarked on FROSTT tensors (scripts/run_cpd.sh) that are
not available offline; these generators stand in for them with the shapes
and value distributions of the named workloads:

  * zipf_tensor_device: per-mode Zipf(s) coordinates over [0, I_n) (rank k
    has probability ~ (k+1)^-s; rows are not permuted, so heavy rows have
    small indices), values lognormal(0,1) drawn in FP32 and summed over
    duplicate coordinates in FP64, exactly `nnz` distinct coordinates.
    Generated on the GPU with torch (plumbing only; not the engine).
  * uniform_tensor_host: distinct uniform coordinates, U(0,1) FP64 values,
    generated with numpy (the small CPU-runnable workload).
"""
import numpy as np


def _zipf_cdf(torch, d, s, device):
    k = torch.arange(1, d + 1, dtype=torch.float64, device=device)
    w = k.pow(-s)
    c = torch.cumsum(w, 0)
    return c / c[-1]


def zipf_tensor_device(nnz, dims, s, seed=0, device="cuda", value_dist="lognormal"):
    """Returns dict(dims, cidx=[int64 CUDA tensors], vals=float64 CUDA tensor)."""
    import torch
    dims = [int(d) for d in dims]
    key_space = 1
    for d in dims:
        key_space *= d
    if key_space >= 2 ** 63:
        raise ValueError("coordinate space too large for 63-bit linear keys")
    if nnz > key_space:
        raise ValueError("more nonzeros than cells")
    g = torch.Generator(device=device).manual_seed(int(seed))
    cdfs = [_zipf_cdf(torch, d, s, device) if s > 0 else None for d in dims]
    mult = []
    m = 1
    for d in reversed(dims):
        mult.append(m)
        m *= d
    mult = list(reversed(mult))

    keys = torch.empty(0, dtype=torch.int64, device=device)
    vals = torch.empty(0, dtype=torch.float64, device=device)
    draw = int(nnz * 1.05) + 1024
    for _ in range(64):
        k = torch.zeros(draw, dtype=torch.int64, device=device)
        for n, d in enumerate(dims):
            if cdfs[n] is None:
                c = torch.randint(0, d, (draw,), generator=g, device=device, dtype=torch.int64)
            else:
                u = torch.rand(draw, dtype=torch.float64, generator=g, device=device)
                c = torch.searchsorted(cdfs[n], u).clamp_(max=d - 1)
            k += c * mult[n]
            del c
        if value_dist == "lognormal":
            v = torch.randn(draw, dtype=torch.float32, generator=g, device=device).exp_().double()
        else:
            v = torch.rand(draw, dtype=torch.float32, generator=g, device=device).double()
        keys = torch.cat([keys, k])
        vals = torch.cat([vals, v])
        del k, v
        uk, inv = torch.unique(keys, sorted=True, return_inverse=True)
        uv = torch.zeros(uk.numel(), dtype=torch.float64, device=device).index_add_(0, inv, vals)
        del inv
        keys, vals = uk, uv
        have = keys.numel()
        if have >= nnz:
            break
        # draw more, scaled by the observed yield of new distinct keys
        draw = int((nnz - have) * 2.0) + 1024
    else:
        raise RuntimeError("could not reach the requested number of distinct coordinates")
    if keys.numel() > nnz:
        pick = torch.randperm(keys.numel(), generator=g, device=device)[:nnz]
        keys, vals = keys[pick], vals[pick]
    else:
        pick = torch.randperm(keys.numel(), generator=g, device=device)
        keys, vals = keys[pick], vals[pick]
    cidx = []
    rem = keys
    for n, mu in enumerate(mult):
        cidx.append(torch.div(rem, mu, rounding_mode="floor"))
        rem = rem - cidx[-1] * mu
    del keys, rem
    return dict(dims=dims, cidx=cidx, vals=vals.contiguous())


def zipf_coo_device(nnz, dims, s, seed=0, device="cuda", chunk=1 << 28, value_dist="uniform"):
    """Per-mode Zipf(s) coordinates drawn chunk by chunk into preallocated
    int64 arrays, without deduplication (coordinates may repeat; the
    MTTKRP sums repeated nonzeros), values U(0,1) (or lognormal) drawn in
    FP32: a generator whose memory is the COO itself, for nonzero counts
    whose deduplication would not fit the device.
    Returns dict(dims, cidx=[int64 CUDA tensors], vals=float64 CUDA tensor)."""
    import torch
    dims = [int(d) for d in dims]
    g = torch.Generator(device=device).manual_seed(int(seed))
    cdfs = [_zipf_cdf(torch, d, s, device) if s > 0 else None for d in dims]
    cidx = [torch.empty(nnz, dtype=torch.int64, device=device) for _ in dims]
    vals = torch.empty(nnz, dtype=torch.float64, device=device)
    for o in range(0, nnz, chunk):
        n = min(chunk, nnz - o)
        for m, d in enumerate(dims):
            if cdfs[m] is None:
                cidx[m][o:o + n] = torch.randint(0, d, (n,), generator=g, device=device, dtype=torch.int64)
            else:
                u = torch.rand(n, dtype=torch.float64, generator=g, device=device)
                cidx[m][o:o + n] = torch.searchsorted(cdfs[m], u).clamp_(max=d - 1)
                del u
        if value_dist == "lognormal":
            vals[o:o + n] = torch.randn(n, dtype=torch.float32, generator=g, device=device).exp_().double()
        else:
            vals[o:o + n] = torch.rand(n, dtype=torch.float32, generator=g, device=device).double()
    return dict(dims=dims, cidx=cidx, vals=vals)


def wide_tensor_device(nnz, dims, s, seed=0, device="cuda"):
    """Distinct coordinates in a key space above 2^63 (keys of more than 64
    bits): per-mode Zipf(s) draws (uniform for s = 0), deduplicated on a
    pair of linear keys (the modes split into two groups whose products stay
    below 2^62), values lognormal(0,1) drawn in FP32 and summed over
    duplicate coordinates in FP64, exactly `nnz` nonzeros in random order.
    Returns dict(dims, cidx=[int64 CUDA tensors], vals=float64 CUDA tensor)."""
    import torch
    dims = [int(d) for d in dims]
    groups, cur, prod = [], [], 1
    for n, d in enumerate(dims):
        if cur and prod * d >= 2 ** 62:
            groups.append(cur)
            cur, prod = [], 1
        cur.append(n)
        prod *= d
    groups.append(cur)
    if len(groups) > 2:
        raise ValueError("modes do not split into two keys below 2^62")
    while len(groups) < 2:
        groups.append([])
    mults = []
    for grp in groups:
        m, ms = 1, {}
        for n in reversed(grp):
            ms[n] = m
            m *= dims[n]
        mults.append(ms)
    g = torch.Generator(device=device).manual_seed(int(seed))
    cdfs = [_zipf_cdf(torch, d, s, device) if s > 0 else None for d in dims]
    k0 = torch.empty(0, dtype=torch.int64, device=device)
    k1 = torch.empty(0, dtype=torch.int64, device=device)
    vals = torch.empty(0, dtype=torch.float64, device=device)
    draw = int(nnz * 1.02) + 1024
    for _ in range(64):
        a = torch.zeros(draw, dtype=torch.int64, device=device)
        b = torch.zeros(draw, dtype=torch.int64, device=device)
        for n, d in enumerate(dims):
            if cdfs[n] is None:
                c = torch.randint(0, d, (draw,), generator=g, device=device, dtype=torch.int64)
            else:
                u = torch.rand(draw, dtype=torch.float64, generator=g, device=device)
                c = torch.searchsorted(cdfs[n], u).clamp_(max=d - 1)
            if n in mults[0]:
                a += c * mults[0][n]
            else:
                b += c * mults[1][n]
            del c
        v = torch.randn(draw, dtype=torch.float32, generator=g, device=device).exp_().double()
        k0, k1, vals = torch.cat([k0, a]), torch.cat([k1, b]), torch.cat([vals, v])
        del a, b, v
        # lexicographic (k0, k1) order by two stable sorts, then runs
        o = torch.sort(k1, stable=True)[1]
        o = o[torch.sort(k0[o], stable=True)[1]]
        k0, k1, vals = k0[o], k1[o], vals[o]
        del o
        first = torch.ones(k0.numel(), dtype=torch.bool, device=device)
        first[1:] = (k0[1:] != k0[:-1]) | (k1[1:] != k1[:-1])
        rid = torch.cumsum(first.to(torch.int64), 0) - 1
        nu = int(rid[-1].item()) + 1
        vals = torch.zeros(nu, dtype=torch.float64, device=device).index_add_(0, rid, vals)
        k0, k1 = k0[first], k1[first]
        del first, rid
        if nu >= nnz:
            break
        draw = int((nnz - nu) * 2.0) + 1024
    else:
        raise RuntimeError("could not reach the requested number of distinct coordinates")
    pick = torch.randperm(k0.numel(), generator=g, device=device)[:nnz]
    k0, k1, vals = k0[pick], k1[pick], vals[pick]
    cidx = [None] * len(dims)
    for key, ms in ((k0, mults[0]), (k1, mults[1])):
        rem = key
        for n in sorted(ms, key=lambda q: -ms[q]):
            cidx[n] = torch.div(rem, ms[n], rounding_mode="floor")
            rem = rem - cidx[n] * ms[n]
    return dict(dims=dims, cidx=cidx, vals=vals.contiguous())


def uniform_tensor_host(nnz, dims, seed=0):
    """Distinct uniform coordinates and U(0,1) FP64 values (numpy)."""
    rng = np.random.default_rng(seed)
    dims = [int(d) for d in dims]
    mult = np.cumprod([1] + dims[::-1][:-1])[::-1].astype(np.int64)
    total = int(np.prod(np.array(dims, dtype=np.float64)))
    lin = rng.choice(total, size=nnz, replace=False) if total < 50 * nnz else np.unique(
        rng.integers(0, total, size=int(nnz * 1.2) + 16))
    while len(lin) < nnz:
        lin = np.unique(np.concatenate([lin, rng.integers(0, total, size=nnz)]))
    lin = rng.permutation(lin)[:nnz]
    cidx = np.zeros((len(dims), nnz), dtype=np.uint64)
    rem = lin.astype(np.int64)
    for n, mu in enumerate(mult):
        cidx[n] = (rem // mu).astype(np.uint64)
        rem = rem % mu
    vals = rng.random(nnz)
    return dict(dims=dims, cidx=cidx, vals=vals)


def batch_tensors_device(count=512, seed=0, device="cuda", median_nnz=200_000, nnz_range=(10_000, 2_000_000),
                         dim_range=(100, 50_000), ranks=(8, 16, 32), nmodes=3):
    """Many small 3-mode tensors of uneven size (the batched CP-ALS
    workload): nnz lognormal(log median, 1) clipped to nnz_range and to half
    the tensor's cells, each mode length uniform in dim_range, uniform
    coordinates, FP32 U(0,1) values, rank drawn from `ranks`.  Returns a list
    of dict(dims, cidx, vals, rank)."""
    rng = np.random.default_rng(int(seed))
    out = []
    for i in range(count):
        dims = [int(x) for x in rng.integers(dim_range[0], dim_range[1] + 1, size=nmodes)]
        cells = int(np.prod(np.array(dims, dtype=np.float64)))
        nnz = int(np.exp(rng.normal(np.log(median_nnz), 1.0)))
        nnz = int(min(max(nnz, nnz_range[0]), nnz_range[1], cells // 2))
        X = zipf_tensor_device(nnz, dims, 0.0, seed=int(seed) * 100_003 + i, device=device, value_dist="uniform")
        X["rank"] = int(rng.choice(ranks))
        out.append(X)
    return out
