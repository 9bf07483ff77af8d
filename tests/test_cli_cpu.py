"""The command line (esl_cli, the reference's cuda/src/main.cpp:159-312) without a GPU:
argument errors are reported before any device work, with the reference's messages."""
import os
import subprocess

import pytest

from paraexastolog_b200 import build as B


@pytest.fixture(scope="module")
def cli():
    B.build()
    assert os.path.exists(B.CLI)
    return B.CLI


def _run(cli, *args):
    p = subprocess.run([cli, *args], capture_output=True, text=True, timeout=60)
    return p.returncode, p.stdout, p.stderr


def test_usage_without_bnet_file(cli):
    rc, out, err = _run(cli)
    assert rc == 1 and out == "" and "usage: esl_cli -f BNET_FILE" in err


def test_reference_messages(cli):
    rc, _, err = _run(cli, "-f", "x.bnet", "-i", "RANDOM")
    assert rc == 1 and err.startswith("RANDOM initial state distribution not implemented") and "usage" not in err
    rc, _, err = _run(cli, "-f", "x.bnet", "-t", "GAMMA")
    assert rc == 1 and err.startswith("Bad transition distribution type") and "usage" in err
    rc, _, err = _run(cli, "-f", "x.bnet", "--initial-fixed-prob", "1.5")
    assert rc == 1 and err.startswith("Bad fixed initial states probability")


@pytest.mark.parametrize("bad", ["x_A=1", "u_A", "u_A=x", "uA=1"])
def test_bad_transition_rates(cli, bad):
    rc, _, err = _run(cli, "-f", "x.bnet", "--trans-rates", bad)
    assert rc == 1 and "usage" in err


@pytest.mark.parametrize("bad", ["A=2", "A", "A=01"])
def test_bad_fixed_list(cli, bad):
    rc, _, err = _run(cli, "-f", "x.bnet", "--initial-fixed-list", bad)
    assert rc == 1 and "usage" in err


@pytest.mark.parametrize("bad", ["-1", "nan", "1e30", "2.5", "x"])
def test_bad_seed(cli, bad):
    rc, _, err = _run(cli, "-f", "x.bnet", "--seed", bad)
    assert rc == 1 and "usage" in err
