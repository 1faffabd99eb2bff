"""Tests of the cpd64 command-line driver (host/cpd64.cpp).

CPU: argument handling, the FROSTT .tns parser (src/sptensor.cpp:74-160
semantics: '#' comments and blank lines skipped, 1-based indices, each mode
length the largest index) and the binary writer (src/sptensor.cpp:56-68),
checked through `-f 1`, which writes <input>.bin before any GPU work.
GPU: CP-ALS output lines, the -c -p MTTKRP check, the -p benchmark line and
the seeded random initialisation against the reference's (golden fixture).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG_DIR

CPD64 = os.path.join(PKG_DIR, "bin", "cpd64")


def run(args, env=None, timeout=300):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([CPD64] + args, capture_output=True, text=True, timeout=timeout, env=e)


def write_tns(path, cidx, vals, comments=True):
    with open(path, "w") as f:
        if comments:
            f.write("# a comment line\n\n")
        for i in range(cidx.shape[1]):
            f.write(" ".join(str(int(c) + 1) for c in cidx[:, i]) + " %.17g\n" % vals[i])
            if comments and i == 3:
                f.write("# another comment\n")


def read_bin(path):
    with open(path, "rb") as f:
        nm = int(np.frombuffer(f.read(8), dtype=np.uint64)[0])
        dims = np.frombuffer(f.read(8 * nm), dtype=np.uint64)
        nnz = int(np.frombuffer(f.read(8), dtype=np.uint64)[0])
        cidx = np.frombuffer(f.read(8 * nm * nnz), dtype=np.uint64).reshape(nm, nnz)
        vals = np.frombuffer(f.read(8 * nnz), dtype=np.float64)
    return dims, cidx, vals


def test_help_and_version():
    r = run(["-h"])
    assert r.returncode == 0 and "--max-block-size" in r.stderr
    r = run(["-v"])
    assert r.returncode == 0 and "blco_b200" in r.stdout


def test_tns_parser_and_binary_writer(tmp_path):
    rng = np.random.default_rng(3)
    dims = [7, 30, 5]
    lin = rng.choice(7 * 30 * 5, size=200, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    vals = rng.random(200)
    p = str(tmp_path / "x.tns")
    write_tns(p, cidx, vals)
    r = run(["-i", p, "-f", "1"])
    # no -k: the engine refuses the CPU path after reading and writing the file
    assert r.returncode == 1 and "pass -k" in r.stderr
    d, c, v = read_bin(p + ".bin")
    assert list(d) == [int(cidx[n].max()) + 1 for n in range(3)]
    assert np.array_equal(c, cidx) and np.array_equal(v, vals)


def test_selector_file_errors(tmp_path):
    p = str(tmp_path / "x.tns")
    write_tns(p, np.array([[0, 1], [1, 0], [0, 1]], dtype=np.uint64), np.array([1.0, 2.0]), comments=False)
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\x01\x00")
    r = run(["-i", p, "-k", "21", "--host-load", "--selector", str(bad)])
    assert r.returncode == 1 and "selector" in r.stderr
    r = run(["-i", p, "-k", "21", "--host-load", "--selector", str(tmp_path / "missing.bin")])
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_precision_flag_errors():
    r = run(["--precision", "fp16"])
    assert r.returncode == 1 and "Invalid -precision" in r.stderr
    r = run(["--precision", "mixed", "-c", "-i", "missing.tns"])
    assert r.returncode == 1 and "the -c / -p MTTKRP runs are FP64" in r.stderr
    r = run(["-h"])
    assert "--precision" in r.stderr


def test_tns_rejects_bad_input(tmp_path):
    p = str(tmp_path / "bad.tns")
    with open(p, "w") as f:
        f.write("1 2 3 1.0\n0 1 1 2.0\n")
    r = run(["-i", p, "-k", "10", "--host-load"])
    assert r.returncode == 1 and "1-based" in r.stderr
    r = run(["-i", str(tmp_path / "missing.tns"), "-k", "10"])
    assert r.returncode == 1 and "cannot open" in r.stderr
    r = run(["-i", str(tmp_path / "missing.tns"), "-k", "10", "--host-load"])
    assert r.returncode == 1 and "cannot open" in r.stderr
    r = run(["-k", "10"])
    assert r.returncode == 1


@pytest.mark.gpu
def test_cli_cpals_lines_and_export(tmp_path):
    rng = np.random.default_rng(4)
    dims = [40, 30, 20]
    lin = rng.choice(40 * 30 * 20, size=3000, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    vals = rng.random(3000)
    p = str(tmp_path / "t.tns")
    write_tns(p, cidx, vals, comments=False)
    out = str(tmp_path / "model")
    r = run(["-i", p, "-k", "10", "-r", "4", "-m", "5", "-e", "0", "-x", "7", "-o", out])
    assert r.returncode == 0, r.stderr
    iters = [l for l in r.stdout.splitlines() if l.startswith("--> Iter")]
    assert len(iters) == 5
    assert "Final fit:" in r.stdout
    for n in range(3):
        with open(f"{out}.{n}.out") as f:
            lines = f.read().split()
        assert lines[:2] == ["matrix", "2"] and int(lines[2]) == dims[n] and int(lines[3]) == 4
        assert len(lines) == 4 + dims[n] * 4
    with open(f"{out}.lambda.out") as f:
        assert f.read().split()[:3] == ["vector", "1", "4"]


@pytest.mark.gpu
def test_cli_gpu_loader_matches_host_loader(tmp_path):
    """cpd64 parses .tns files on the GPU by default; the fits equal those of
    the host loader (--host-load) on the same file and seed."""
    rng = np.random.default_rng(9)
    dims = [60, 50, 40]
    lin = rng.choice(60 * 50 * 40, size=6000, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    p = str(tmp_path / "g.tns")
    write_tns(p, cidx, rng.random(6000))
    outs = []
    for extra in ([], ["--host-load"]):
        r = run(["-i", p, "-k", "10", "-r", "6", "-m", "5", "-e", "0", "-x", "4"] + extra)
        assert r.returncode == 0, r.stderr
        outs.append([l for l in r.stdout.splitlines() if l.startswith("--> Iter") or l.startswith("Final fit")])
        assert "NNZ             = 6000" in r.stderr
    strip = lambda ls: [l.split("time =")[0] for l in ls]
    assert strip(outs[0]) == strip(outs[1])


@pytest.mark.gpu
def test_cli_random_init_matches_reference(tmp_path):
    """-m 0 exports the initial model: it must equal the reference's
    KruskalModelRandomInit for the same seed and thread count."""
    g = dict(np.load(os.path.join(GOLDEN, "init_t3.npz")))
    dims = [7, 13, 5]
    # a tensor whose mode lengths are 7 x 13 x 5 (largest indices present)
    cidx = np.array([[6, 0, 3], [12, 5, 0], [4, 1, 2]], dtype=np.uint64)
    p = str(tmp_path / "i.tns")
    write_tns(p, cidx, np.array([1.0, 2.0, 3.0]), comments=False)
    out = str(tmp_path / "init")
    r = run(["-i", p, "-k", "10", "-r", "6", "-m", "0", "-x", "12345", "-o", out], env={"OMP_NUM_THREADS": "3"})
    assert r.returncode == 0, r.stderr
    for n in range(3):
        with open(f"{out}.{n}.out") as f:
            vals = np.array([float(x) for x in f.read().split()[4:]])
        got = vals.reshape(6, dims[n]).T  # written column by column
        assert np.allclose(got, g[f"f{n}"], rtol=0, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["1", "2", "3", "10", "13", "20", "21"])
def test_cli_check_mode(tmp_path, kernel):
    rng = np.random.default_rng(5)
    dims = [50, 60, 70]
    lin = rng.choice(50 * 60 * 70, size=5000, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    p = str(tmp_path / "c.tns")
    write_tns(p, cidx, rng.random(5000), comments=False)
    sel = ["--selector", os.path.join(PKG_DIR, "selector", "selector_params.bin")] if kernel == "21" else []
    for mode in ("0", "2"):
        r = run(["-i", p, "-k", kernel, "-c", "-p", "-t", mode, "-r", "8", "-x", "1"] + sel)
        assert r.returncode == 0, r.stderr
        assert r.stderr.count("Results of mttkrp_blco_dev is correct") == 3, r.stderr


@pytest.mark.gpu
def test_cli_bench_and_streamed(tmp_path):
    rng = np.random.default_rng(6)
    dims = [100, 90, 80]
    lin = rng.choice(100 * 90 * 80, size=20000, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    p = str(tmp_path / "b.tns")
    write_tns(p, cidx, rng.random(20000), comments=False)
    r = run(["-i", p, "-k", "1", "-p", "-t", "1", "-m", "3", "-r", "16"])
    assert r.returncode == 0 and "Total time for MTTKRP:" in r.stdout
    r = run(["-i", p, "-k", "2", "-c", "-p", "-t", "1", "-r", "16", "--stream-data", "--max-block-size", "3000"])
    assert r.returncode == 0, r.stderr
    assert r.stderr.count("is correct") == 3
    # CP-ALS with the stream in host memory follows the resident run
    fits = []
    for extra in ([], ["--stream-data", "--max-block-size", "3000"]):
        r = run(["-i", p, "-k", "10", "-r", "8", "-m", "4", "-e", "0", "-x", "3"] + extra)
        assert r.returncode == 0, r.stderr
        fits.append([float(l.split("f = ")[1].split()[0]) for l in r.stdout.splitlines() if l.startswith("--> Iter")])
    assert len(fits[0]) == 4 and np.allclose(fits[0], fits[1], rtol=0, atol=2e-6)
    # CP-ALS with the stream in host memory follows the resident run
    fits = []
    for extra in ([], ["--stream-data", "--max-block-size", "3000"]):
        r = run(["-i", p, "-k", "10", "-r", "8", "-m", "4", "-e", "0", "-x", "3"] + extra)
        assert r.returncode == 0, r.stderr
        fits.append([float(l.split("f = ")[1].split()[0]) for l in r.stdout.splitlines() if l.startswith("--> Iter")])
    assert len(fits[0]) == 4 and np.allclose(fits[0], fits[1], rtol=0, atol=2e-6)


@pytest.mark.gpu
def test_cli_wide_keys(tmp_path):
    """A tensor whose coordinates need 69 key bits (the reference's cpd128
    case): CP-ALS through the GPU and the host loader give the same fits,
    and the -c check of every mode's MTTKRP passes."""
    rng = np.random.default_rng(17)
    dims = [9000, 8500, 8200, 8192, 8300]
    c = np.stack([rng.integers(0, d, size=6000, dtype=np.uint64) for d in dims])
    cidx = np.unique(c, axis=1)
    # every mode's largest index present, so the loaders find these lengths
    cidx[:, 0] = np.array(dims, dtype=np.uint64) - 1
    cidx = np.unique(cidx, axis=1)
    p = str(tmp_path / "w.tns")
    write_tns(p, cidx, rng.random(cidx.shape[1]))
    outs = []
    for extra in ([], ["--host-load"]):
        r = run(["-i", p, "-k", "10", "-r", "4", "-m", "4", "-e", "0", "-x", "3"] + extra)
        assert r.returncode == 0, r.stderr
        outs.append([l.split("time =")[0] for l in r.stdout.splitlines()
                     if l.startswith("--> Iter") or l.startswith("Final fit")])
    assert len(outs[0]) == 5 and outs[0] == outs[1]
    for mode in ("0", "4"):
        r = run(["-i", p, "-k", "10", "-c", "-p", "-t", mode, "-r", "8", "-x", "1"])
        assert r.returncode == 0, r.stderr
        # one verification line per mode
        assert r.stderr.count("Results of mttkrp_blco_dev is correct") == 5, r.stderr


@pytest.mark.gpu
def test_cli_mixed_precision_cpals(tmp_path):
    """--precision mixed runs the chosen form: the fit follows the FP64
    run's within the chosen form's 1e-5 bound."""
    rng = np.random.default_rng(23)
    dims = [80, 60, 40]
    lin = rng.choice(80 * 60 * 40, size=20000, replace=False)
    cidx = np.array(np.unravel_index(lin, dims), dtype=np.uint64)
    p = str(tmp_path / "m.tns")
    write_tns(p, cidx, rng.random(20000), comments=False)
    fits = {}
    for prec in ("fp64", "mixed"):
        r = run(["-i", p, "-k", "10", "-r", "8", "-m", "6", "-e", "0", "-x", "5", "--precision", prec])
        assert r.returncode == 0, r.stderr
        line = [l for l in r.stdout.splitlines() if l.startswith("Final fit")][0]
        fits[prec] = float(line.split(":")[1])
    assert abs(fits["mixed"] - fits["fp64"]) <= 1e-5
