"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own CPU code, compiled from its sources by
`make -C oracle ref` into oracle/_ref/libblco_ref.so:
  * gen_blcotensor_host<uint64> (include/blco.hpp:196-331) -> BLCO coords,
    values, masks, positions, block offsets and block coordinates;
  * the sequential COO MTTKRP (include/cpd.hpp:510-544) for every mode;
  * KruskalModelRandomInit (src/kruskal_model.cpp:93-110) under a stated
    OpenMP thread count.
The w128_* cases come from the cpd128 build's encoder,
gen_blcotensor_host<unsigned __int128>, on tensors whose coordinates need
more than 64 key bits (several blocks with non-zero block coordinates).
Inputs are seeded synthetic tensors (unique coordinates; the reference leaves
the order of duplicate coordinates unspecified).  Usage, from the repo root:

    make -C oracle && make -C oracle ref
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --wide     # only the w128_* fixtures
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402


def unique_coords(rng, dims, nnz, zipf=None):
    """nnz distinct coordinates; zipf=s draws each mode from a Zipf law
    P(k) ~ 1/(k+1)^s over [0, dim), otherwise uniform."""
    dims = [int(d) for d in dims]
    seen = set()
    out = []
    while len(out) < nnz:
        m = 2 * (nnz - len(out)) + 16
        cols = []
        for d in dims:
            if zipf is None:
                cols.append(rng.integers(0, d, size=m))
            else:
                w = 1.0 / np.arange(1, d + 1, dtype=np.float64) ** zipf
                cols.append(rng.choice(d, size=m, p=w / w.sum()))
        for t in zip(*cols):
            if t not in seen:
                seen.add(t)
                out.append(t)
                if len(out) == nnz:
                    break
    return np.array(out, dtype=np.uint64).T.copy()


def formula_factors(dims, rank):
    """Deterministic factor matrices, recomputed by the tests instead of
    being stored: U_m[i, r] = 0.25 + ((i*2654435761 + r*40503 + m*97) mod
    1000003) / 1000003."""
    out = []
    for m, d in enumerate(dims):
        i = np.arange(int(d), dtype=np.int64)[:, None]
        r = np.arange(rank, dtype=np.int64)[None, :]
        out.append(0.25 + ((i * 2654435761 + r * 40503 + m * 97) % 1000003) / 1000003.0)
    return out


CASES = [
    # name, dims, nnz, max_block_size, rank, zipf
    ("kat_5x3x9", [5, 3, 9], None, 4, 4, None),
    ("u3_small", [37, 1000, 5], 2000, 300, 8, None),
    ("u3_pow2", [64, 65, 2], 1500, 0, 16, None),
    ("u4", [100, 20, 300, 7], 3000, 1024, 8, None),
    ("u5", [9, 17, 33, 65, 129], 2500, 700, 4, None),
    ("zipf3", [5000, 4000, 300], 4000, 1000, 16, 1.1),
    ("one_nnz", [10, 10, 10], 1, 0, 3, None),
    ("ties_equal_bits", [16, 16, 16], 800, 256, 5, None),
    ("long_short", [1 << 20, 3, 1 << 12], 3000, 0, 16, None),
]


WIDE_CASES = [
    # name, dims, nnz, max_block_size, rank (0: encoder only), zipf
    ("w128_5mode", [9000, 8500, 8200, 8192, 8300], 3000, 100, 4, None),
    ("w128_4mode", [131073, 131072, 100000, 70000], 4000, 0, 8, None),
    ("w128_zipf5", [9000, 9000, 9000, 70000, 600], 3000, 64, 6, 0.9),
    ("w128_long", [(1 << 31) + 5, 1 << 31, 17], 2500, 7, 0, None),
]


def ref_mttkrp(dims, cidx, vals, factors, m):
    """The reference COO MTTKRP (include/cpd.hpp:510-544) of mode m; the
    reference accumulates into U[m], so it gets a zeroed copy."""
    import ctypes
    fs = [f.copy() for f in factors]
    fs[m][:] = 0.0
    arrs = [np.ascontiguousarray(f) for f in fs]
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    d64 = np.ascontiguousarray(dims, dtype=np.uint64)
    po.ref_lib().ref_mttkrp_coo(ctypes.c_int(len(dims)), d64.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                ctypes.c_uint64(cidx.shape[1]),
                                cidx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                ctypes.c_int(factors[0].shape[1]), ptrs, ctypes.c_int(m))
    return arrs[m]


def wide_main():
    rng = np.random.default_rng(20240602)
    index = []
    for name, dims, nnz, B, rank, zipf in WIDE_CASES:
        cidx = unique_coords(rng, dims, nnz, zipf)
        vals = rng.uniform(0.0, 1.0, size=cidx.shape[1])
        r = po.ref_blco_encode128(dims, cidx, vals, B)
        payload = dict(dims=np.array(dims, dtype=np.uint64), cidx=cidx, vals=vals,
                       max_block_size=np.uint64(B), rank=np.int64(rank),
                       coords=r["coords"], out_vals=r["vals"], mode_masks=r["mode_masks"],
                       mode_pos=r["mode_pos"], block_offsets=r["block_offsets"],
                       block_coords=r["block_coords"])
        if rank:
            factors = formula_factors(dims, rank)
            for m in range(len(dims)):
                payload[f"mttkrp{m}"] = ref_mttkrp(dims, cidx, vals, factors, m)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **payload)
        index.append(dict(name=name, dims=dims, nnz=int(cidx.shape[1]), max_block_size=B, rank=rank,
                          zipf=zipf, nblocks=int(r["nblocks"]), key_bits=int(sum(int(d - 1).bit_length()
                                                                                   for d in dims))))
    return index


def kat_inputs():
    pts = [(4, 2, 8, 1.0), (0, 0, 0, 2.0), (1, 2, 3, 3.0), (3, 1, 0, 4.0), (2, 0, 5, 5.0), (0, 1, 7, 6.0)]
    cidx = np.array([[p[n] for p in pts] for n in range(3)], dtype=np.uint64)
    vals = np.array([p[3] for p in pts], dtype=np.float64)
    return cidx, vals


def main():
    if po.ref_lib() is None:
        sys.exit("oracle/_ref not built: run `make -C oracle ref` first")
    if "--wide" in sys.argv[1:]:
        path = os.path.join(HERE, "index.json")
        with open(path) as f:
            doc = json.load(f)
        doc["wide_cases"] = wide_main()
        with open(path, "w") as f:
            json.dump(doc, f, indent=1)
        print("wrote", len(doc["wide_cases"]), "wide cases")
        return
    rng = np.random.default_rng(20240601)
    index = []
    for name, dims, nnz, B, rank, zipf in CASES:
        if nnz is None:
            cidx, vals = kat_inputs()
        else:
            cidx = unique_coords(rng, dims, nnz, zipf)
            vals = rng.uniform(0.0, 1.0, size=cidx.shape[1])
        r = po.ref_blco_encode(dims, cidx, vals, B)
        factors = formula_factors(dims, rank)
        mttkrp = []
        for m in range(len(dims)):
            # the reference accumulates into U[m]; pass a copy with U[m] = 0
            fs = [f.copy() for f in factors]
            fs[m][:] = 0.0
            R = po.ref_lib()
            import ctypes
            arrs = [np.ascontiguousarray(f) for f in fs]
            ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
            d64 = np.ascontiguousarray(dims, dtype=np.uint64)
            R.ref_mttkrp_coo(ctypes.c_int(len(dims)), d64.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                             ctypes.c_uint64(cidx.shape[1]),
                             cidx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                             vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             ctypes.c_int(rank), ptrs, ctypes.c_int(m))
            mttkrp.append(arrs[m])
        payload = dict(dims=np.array(dims, dtype=np.uint64), cidx=cidx, vals=vals,
                       max_block_size=np.uint64(B), rank=np.int64(rank),
                       coords=r["coords"], out_vals=r["vals"], mode_masks=r["mode_masks"],
                       mode_pos=r["mode_pos"], block_offsets=r["block_offsets"],
                       block_coords=r["block_coords"])
        for m in range(len(dims)):
            payload[f"mttkrp{m}"] = mttkrp[m]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **payload)
        index.append(dict(name=name, dims=dims, nnz=int(cidx.shape[1]), max_block_size=B,
                          rank=rank, zipf=zipf, nblocks=int(r["nblocks"])))

    # KruskalModelRandomInit under several OpenMP thread counts: run the
    # reference in child processes with OMP_NUM_THREADS set.
    inits = []
    for nthreads in (1, 3, 8):
        env = dict(os.environ, OMP_NUM_THREADS=str(nthreads))
        code = ("import sys, numpy as np, ctypes; sys.path.insert(0, %r); import pyoracle as po;"
                "dims=np.array([7,13,5],dtype=np.uint64); rank=6;"
                "fs=[np.zeros((int(d),rank)) for d in dims]; lam=np.zeros(rank);"
                "p=(ctypes.c_void_p*3)(*[f.ctypes.data for f in fs]);"
                "po.ref_lib().ref_kruskal_random_init(ctypes.c_int(3), dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),"
                "ctypes.c_int(rank), ctypes.c_uint(12345), p, lam.ctypes.data_as(ctypes.POINTER(ctypes.c_double)));"
                "np.savez_compressed(%r, f0=fs[0], f1=fs[1], f2=fs[2], lam=lam)")
        path = os.path.join(HERE, f"init_t{nthreads}.npz")
        subprocess.run([sys.executable, "-c", code % (os.path.join(ROOT, "oracle"), path)],
                       env=env, check=True, stdout=subprocess.DEVNULL)
        inits.append(dict(file=f"init_t{nthreads}.npz", nthreads=nthreads, seed=12345,
                          dims=[7, 13, 5], rank=6))
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(dict(generator="tests/golden/make_golden.py", source="reference CPU code via oracle/_ref",
                       cases=index, inits=inits, wide_cases=wide_main()), f, indent=1)
    print("wrote", len(index), "cases and", len(inits), "init fixtures")


if __name__ == "__main__":
    main()
