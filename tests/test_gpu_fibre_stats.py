"""GPU: the compressed-fibre copy's counts against a count made here.

`blco_tensor_fibre_stats` reports what a mode's copy holds: its fibre mode
(the shortest other mode, the first of equal lengths), the nonzeros in
fibres of two or more, the single-nonzero fibres, the fibres of two or more
and the factor rows one MTTKRP of the mode gathers ((nmodes - 2) per fibred
nonzero, one per fibre, nmodes - 1 per single-nonzero fibre).  The benchmark
divides that row count by the MTTKRP's time for its gather rate.  Here numpy
groups the COO coordinates by (row of the mode, index of the fibre mode) and
the two must agree exactly: they are integer counts.
"""
import numpy as np
import pytest

from conftest import unique_coords

pytestmark = pytest.mark.gpu


def expected_stats(cidx, dims, mode):
    n = len(dims)
    fm = min((k for k in range(n) if k != mode), key=lambda k: dims[k])
    key = cidx[mode].astype(np.uint64) * np.uint64(dims[fm]) + cidx[fm].astype(np.uint64)
    _, counts = np.unique(key, return_counts=True)
    single = int((counts == 1).sum())
    fibres = int((counts >= 2).sum())
    fibred = int(counts[counts >= 2].sum())
    return dict(fibre_mode=fm, fibred_nnz=fibred, single_nnz=single, fibres=fibres,
                rows_gathered=fibred * (n - 2) + fibres + single * (n - 1))


@pytest.mark.parametrize("dims,nnz,zipf", [
    ([2000, 1500, 40], 60_000, 1.1),         # short third mode: many repeated fibres
    ([300, 300, 300], 20_000, None),         # equal lengths: the first other mode
    ([500, 64, 900, 64], 40_000, 0.8),       # 4 modes, tied shortest modes
    ([40, 30, 20, 10, 50], 30_000, 1.2),     # 5 modes
    ([100_000, 80_000, 5_000], 3_000, None),  # almost every fibre a single nonzero
])
def test_fibre_stats_match_numpy(blco, dims, nnz, zipf):
    rng = np.random.default_rng(nnz + len(dims))
    cidx = unique_coords(rng, dims, nnz, zipf=zipf)
    vals = rng.random(nnz)
    t = blco.Tensor.encode(dims, cidx, vals)
    for m in range(len(dims)):
        got = t.fibre_stats(m)
        want = expected_stats(cidx, dims, m)
        assert got == want, (m, got, want)
        assert got["fibred_nnz"] + got["single_nnz"] == nnz
    t.free()
