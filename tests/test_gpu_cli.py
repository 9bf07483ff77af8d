"""The command line (esl_cli) on the reference's known-answer cases, and its .symb files.

- Output: the reference's print_final_state format (cuda/src/solver.cu:336-372); the
  states above 1e-12 are the golden nonzero states, with values within the goldens'
  tolerance (128 FLT_EPS, or 1e-7 for the mammal case).
- .symb: the reference's layout (cuda/src/persistent_solution.cu:31-95): 16 size_t
  sizes, then int32 / FP32 arrays; the table equals esl_table_build's CSC, the order
  and SCC offsets equal esl_net_export's, the terminal kernels equal esl_solve's R.  A
  second run reads the file and prints the same; a run with other rates rewrites it.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from paraexastolog_b200 import build as B
from tests.helpers import FLT_EPS

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def esl():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import paraexastolog_b200 as E
    E.lib()
    return E


@pytest.fixture(scope="module")
def cli():
    B.build()
    return B.CLI


def _args(c):
    a = []
    if c.get("fixed"):
        a += ["--initial-fixed-list", ",".join(f"{n}={v}" for n, v in zip(c["fixed"], c["values"]))]
    rates = [f"u_{k}={v}" for k, v in (c.get("up") or {}).items()] + \
            [f"d_{k}={v}" for k, v in (c.get("down") or {}).items()]
    if rates:
        a += ["--trans-rates", ",".join(rates)]
    return a


def _parse(out, names):
    res = {}
    for line in out.strip().splitlines():
        label, val = line.rsplit(" ", 1)
        s = 0
        if label != "<nil>":
            for nm in label.split(" --- "):
                s |= 1 << names.index(nm)
        res[s] = float(val)
    return res


def _run(cli, path, *args):
    p = subprocess.run([cli, "-f", str(path), *args], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    return p.stdout


@pytest.mark.parametrize("name", ["solver.toy", "solver.kras", "rates.toy", "zero_rate.toy", "solver.mammal",
                                  "solver.zanudo"])
def test_cli_goldens(esl, cli, goldens, tmp_path, name):
    c = goldens["cases"][name]
    text = goldens["models"][c["model"]]
    path = tmp_path / "model.bnet"
    path.write_text(text)
    names = esl.Model.parse(text).names
    got = _parse(_run(cli, path, *_args(c)), names)
    big = sorted(s for s, v in got.items() if v > 1e-12)
    assert big == c["nonzero_indices"]
    tol = 1e-7 if c.get("tolerance") == "1e-7" else 128 * FLT_EPS
    data = c["nonzero_data"] if c.get("nonzero_data") is not None else [c["nonzero_data_each"]] * len(big)
    np.testing.assert_allclose([got[s] for s in big], data, atol=tol, rtol=0)


def _read_symb(path):
    raw = open(path, "rb").read()
    sizes = struct.unpack("16Q", raw[:128])
    kinds = ["i", "i", "i", "i", "i", "i", "f", "i", "i", "f", "i", "i", "f", "i", "i", "f"]
    out, off = [], 128
    for n, k in zip(sizes, kinds):
        dt = np.int32 if k == "i" else np.float32
        out.append(np.frombuffer(raw, dt, n, off))
        off += 4 * n
    assert off == len(raw)
    return sizes, out


def test_cli_symbolic_file(esl, cli, goldens, tmp_path):
    ctx = esl.Context(0)
    text = goldens["models"]["krasmodel15vars.bnet"]
    path = tmp_path / "kras.bnet"
    path.write_text(text)
    symb = tmp_path / "kras.symb"
    first = _run(cli, path, "-s")
    assert symb.exists()
    sizes, (rows, cols, indptr, order, toff, ntoff, rates, st_ip, st_idx, st_data,
            snt_ip, snt_idx, snt_data, inv_ip, inv_idx, inv_data) = _read_symb(symb)
    assert sizes[13:] == (0, 0, 0)
    m = esl.Model.parse(text)
    r = m.rates_uniform()
    ip, rw, cl = esl.table(ctx, m, r)
    assert np.array_equal(indptr, ip.cpu().numpy()) and np.array_equal(rows, rw.cpu().numpy())
    assert np.array_equal(cols, cl.cpu().numpy())
    net = esl.Net.build(ctx, m, r)
    o, offs, _, _ = net.export()
    offs = offs.cpu().numpy()
    assert np.array_equal(order, o.cpu().numpy())
    assert np.array_equal(toff, offs[: net.T + 1]) and np.array_equal(ntoff, offs[net.T:])
    assert np.array_equal(rates, r.astype(np.float32))
    x0 = m.initial_state(ctx)
    res = esl.solve(ctx, net, r, x0, want_R=True)
    assert np.array_equal(st_ip, offs[: net.T + 1]) and np.array_equal(st_idx, order[: net.terminal_states])
    np.testing.assert_allclose(st_data, res.R.cpu().numpy(), rtol=1e-6, atol=0)
    assert snt_ip[-1] == snt_idx.size == snt_data.size
    stamp = os.path.getmtime(symb)
    # the stored table replaces the table construction; same rates: file kept
    assert _run(cli, path, "-s") == first
    assert os.path.getmtime(symb) == stamp
    # other rates: same output as without symbolic data, file rewritten
    other = ["--trans-rates", "u_" + m.names[0] + "=2.5"]
    assert _run(cli, path, "-s", *other) == _run(cli, path, *other)
    _, arrays = _read_symb(symb)
    assert arrays[6][0] == np.float32(2.5)


def test_cli_turns_away_a_damaged_symbolic_file(esl, cli, goldens, tmp_path):
    # a stored table whose column pointers do not end at its edge count is not
    # uploaded (the kernels that read it index rows through them unchecked): the run
    # builds the table itself, prints what a run without -s prints and rewrites the file
    text = goldens["models"]["krasmodel15vars.bnet"]
    path = tmp_path / "kras.bnet"
    path.write_text(text)
    symb = tmp_path / "kras.symb"
    plain = _run(cli, path)
    assert _run(cli, path, "-s") == plain
    good = symb.read_bytes()
    sizes, arrays = _read_symb(symb)
    indptr_last = 128 + 4 * (sizes[0] + sizes[1] + sizes[2] - 1)
    assert struct.unpack_from("<i", good, indptr_last)[0] == arrays[2][-1] == sizes[0]
    bad = bytearray(good)
    struct.pack_into("<i", bad, indptr_last, int(sizes[0]) + 1000)
    symb.write_bytes(bytes(bad))
    assert _run(cli, path, "-s") == plain
    sizes2, arrays2 = _read_symb(symb)
    assert sizes2[:7] == sizes[:7]
    for k in range(7):  # table, order, SCC offsets and rates as first written
        assert np.array_equal(arrays2[k], arrays[k]), k
