"""The .tns loader's decimal conversion (blco_parse_decimal: the code the
GPU runs, compiled for the host) against correctly rounded conversion
(Python's float(), which rounds exactly as strtod does), and the GPU loader
against the host loader (bit-exact encodings).

CPU: every number the conversion decides must be bit-identical to float();
the ones it leaves to strtod must be rare for ordinary inputs.
GPU: files with comments, blank lines, CRLF, tabs, signs, exponents, long
significands and odd spacing, encoded by blco_encode_tns and by blco_encode
from the host loader's arrays.
"""
import os
import random
import struct

import numpy as np
import pytest

from conftest import unique_coords


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _check(blco, text):
    st, v, used = blco.parse_decimal(text)
    if st == 0:
        ref = float(text[:used])
        assert _bits(v) == _bits(ref), (text, v, ref)
    return st


def test_parse_decimal_random_17_digit_values(blco):
    rng = random.Random(1)
    host = 0
    n = 200_000
    for _ in range(n):
        x = rng.random() * 10 ** rng.randint(-30, 30)
        for fmt in ("%.17g", "%.15g", "%.6g", "%.20e", "%r"):
            s = fmt % x if fmt != "%r" else repr(x)
            host += _check(blco, s) == 1
    assert host < 0.001 * n * 5, host


def test_parse_decimal_random_digit_strings(blco):
    rng = random.Random(2)
    for _ in range(100_000):
        nd = rng.randint(1, 19)
        digits = "".join(rng.choice("0123456789") for _ in range(nd))
        dot = rng.randint(0, nd)
        body = digits[:dot] + "." + digits[dot:] if rng.random() < 0.7 else digits
        if body in (".",):
            continue
        exp = rng.choice(["", "e%d" % rng.randint(-330, 310), "E+%d" % rng.randint(0, 40), "e-%d" % rng.randint(0, 40)])
        sign = rng.choice(["", "-", "+"])
        s = sign + body + exp
        st = _check(blco, s)
        assert st in (0, 1)


def test_parse_decimal_edge_forms(blco):
    cases = ["0", "-0", "0.0", ".5", "5.", "+.25e+2", "1e23", "9007199254740993", "2.2250738585072014e-308",
             "4.9e-324", "1.7976931348623157e308", "1e309", "1e-400", "123456789012345678901234567890",
             "0.000000000000000000000000000000000001", "1e", "1e+", "3.25xyz", "  \t 42", "1_0"]
    for c in cases:
        st = _check(blco, c)
        assert st in (0, 1), c
    # exact halfway cases and out-of-range results go to strtod
    assert blco.parse_decimal("1e23")[0] == 1
    assert blco.parse_decimal("9007199254740993")[0] == 1
    assert blco.parse_decimal("1e309")[0] == 1
    assert blco.parse_decimal("4.9e-324")[0] == 1
    for c in ("inf", "-nan", "0x1p3", "Infinity"):
        assert blco.parse_decimal(c)[0] == 1
    for c in ("", "abc", ".", "-", "+e5"):
        assert blco.parse_decimal(c)[0] == 2
    st, v, used = blco.parse_decimal("1e+")
    assert st == 0 and v == 1.0 and used == 1
    st, v, used = blco.parse_decimal("3.25xyz")
    assert st == 0 and v == 3.25 and used == 4


def _write(path, lines):
    with open(path, "w", newline="") as f:
        f.write("".join(lines))


@pytest.mark.gpu
def test_gpu_loader_matches_host_loader(blco, tmp_path):
    rng = np.random.default_rng(3)
    dims = [300, 40, 700, 9]
    nnz = 50_000
    cidx = unique_coords(rng, dims, nnz)
    vals = rng.random(nnz) * 10.0 ** rng.integers(-20, 20, size=nnz)
    pyr = random.Random(4)
    lines = ["# generated\n", "\n"]
    special = {}
    for i in range(nnz):
        sep = pyr.choice([" ", "\t", "  "])
        idx = sep.join(str(int(c) + 1) for c in cidx[:, i])
        v = float(vals[i])
        form = pyr.choice(["%.17g", "%.17e", "%r", "%.25g"])
        s = (form % v) if form != "%r" else repr(v)
        if i % 997 == 0:
            # forms the device leaves to strtod: an exact halfway case, hex
            s = pyr.choice(["1e23", "0x1.8p1"])
            special[i] = float.fromhex(s) if s.startswith("0x") else float(s)
        eol = pyr.choice(["\n", "\r\n", " \n"])
        lines.append(idx + sep + s + eol)
        if pyr.random() < 0.01:
            lines.append(pyr.choice(["# comment\n", "\n", "\r\n"]))
    # the last line without a newline
    lines[-1] = lines[-1].rstrip("\n").rstrip("\r")
    p = str(tmp_path / "t.tns")
    _write(p, lines)
    # what the host loader would read: the same strings through float()
    data = [l for l in lines[2:] if l.strip() and not l.startswith("#")]
    expect_vals = np.array([special.get(i, None) if i in special else float(l.split()[-1])
                            for i, l in enumerate(data)], dtype=np.float64)
    assert len(expect_vals) == nnz
    t_gpu, info = blco.Tensor.encode_tns(p)
    assert info["nmodes"] == 4 and info["nnz"] == nnz
    assert info["dims"] == [int(cidx[n].max()) + 1 for n in range(4)]
    assert info["host_parsed"] >= len(special)
    t_ref = blco.Tensor.encode(info["dims"], cidx, expect_vals)
    a, b = t_gpu.copy_out(), t_ref.copy_out()
    assert np.array_equal(a["coords"], b["coords"])
    assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64))
    t_gpu.free()
    t_ref.free()


@pytest.mark.gpu
def test_gpu_loader_errors(blco, tmp_path):
    p = str(tmp_path / "bad.tns")
    _write(p, ["1 2 3 1.0\n", "2 0 1 2.0\n"])
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode_tns(p)
    assert e.value.status == blco.ERR_INVALID and "line 2" in str(e.value) and "1-based" in str(e.value)
    _write(p, ["1 2 3 1.0\n", "2 x 1 2.0\n"])
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode_tns(p)
    assert "malformed line on line 2" in str(e.value)
    with pytest.raises(blco.BlcoError) as e:
        blco.Tensor.encode_tns(str(tmp_path / "missing.tns"))
    assert e.value.status == blco.ERR_IO


def _edge_files():
    """.tns files whose every line the reference's reader defines
    (src/sptensor.cpp:74-160): comments, empty lines, tabs and runs of
    spaces, leading blanks, signed and exponent and hexadecimal values, long
    significands, CRLF data lines, trailing blanks after the first data line,
    duplicates, one file without a final newline; 3 to 5 modes."""
    rng = np.random.default_rng(31)
    pyr = random.Random(32)
    files = {}
    for name, dims, nnz in (("three", [50, 7, 300], 4000), ("five", [9, 4, 200, 3, 60], 3000),
                            ("one", [5, 5, 5], 1)):
        cidx = unique_coords(rng, dims, nnz)
        if nnz > 1:
            cidx = np.concatenate([cidx, cidx[:, :25]], axis=1)  # duplicates, later in the file
        vals = rng.standard_normal(cidx.shape[1]) * 10.0 ** rng.integers(-12, 12, size=cidx.shape[1])
        lines = ["# a comment line\n", "\n", "#\tanother\n"]
        for i in range(cidx.shape[1]):
            sep = pyr.choice([" ", "\t", "   ", " \t "])
            lead = "" if i == 0 else pyr.choice(["", " ", "\t"])
            idx = sep.join(str(int(c) + 1) for c in cidx[:, i])
            v = float(vals[i])
            s = pyr.choice(["%.17g", "%+.17e", "%.25g", "%.6E", "%r"])
            s = repr(v) if s == "%r" else s % v
            if i % 101 == 7:
                s = pyr.choice(["0x1.8p-3", "-0X1P+4", "1e23", "+.5", "-0.0"])
            eol = "\n" if i == 0 else pyr.choice(["\n", "\r\n", " \n", "\t\n"])
            lines.append(lead + idx + sep + s + eol)
            if pyr.random() < 0.02:
                lines.append(pyr.choice(["# comment\n", "\n"]))
        if name == "five":
            lines[-1] = lines[-1].rstrip("\n").rstrip("\r")
        files[name] = lines
    return files


@pytest.mark.gpu
def test_gpu_loader_matches_reference_reader(blco, tmp_path):
    """blco_encode_tns against the reference's own reader
    (ImportSparseTensor, src/sptensor.cpp:162, built in oracle/_ref) on the
    same files: mode count, lengths, nnz, and the encoding of the reference's
    COO arrays, bit for bit."""
    import pyoracle as po
    if po.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    for name, lines in _edge_files().items():
        p = str(tmp_path / f"{name}.tns")
        _write(p, lines)
        dims, cidx, vals = po.ref_import_tns(p)
        t, info = blco.Tensor.encode_tns(p)
        assert info["nmodes"] == len(dims) and info["dims"] == dims and info["nnz"] == len(vals), name
        ref = blco.Tensor.encode(dims, cidx, vals)
        a, b = t.copy_out(), ref.copy_out()
        assert np.array_equal(a["coords"], b["coords"]), name
        assert np.array_equal(a["vals"].view(np.uint64), b["vals"].view(np.uint64)), name
        t.free()
        ref.free()


def test_reference_reader_on_edge_files(tmp_path):
    """The reference reader (oracle/_ref) on the edge files against a plain
    Python reading of the same lines (split on blanks, float() values, hex
    through float.fromhex): pins the harness the GPU test compares with."""
    import pyoracle as po
    if po.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    for name, lines in _edge_files().items():
        p = str(tmp_path / f"{name}.tns")
        _write(p, lines)
        dims, cidx, vals = po.ref_import_tns(p)
        data = [l.split() for l in lines if len(l) > 1 and not l.startswith("#")]
        want_c = np.array([[int(x) - 1 for x in f[:-1]] for f in data], dtype=np.uint64).T
        want_v = np.array([float.fromhex(f[-1]) if "x" in f[-1].lower() else float(f[-1]) for f in data])
        assert dims == [int(c.max()) + 1 for c in want_c], name
        assert np.array_equal(cidx, want_c), name
        assert np.array_equal(vals.view(np.uint64), want_v.view(np.uint64)), name
