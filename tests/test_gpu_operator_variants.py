"""The two kernel families of the level sweep's Schur operator give the oracle's answer.

FP64 grid groups above 2,048 rows run 32-system tiles with the paired-row kernels by
default (a half warp per row, two systems per lane, `k_sw_elim_pr` / `k_sw_apply_pr`);
`ESL_SWEEP_OP=reg` selects one system per lane (`k_sw_elim` / `k_sw_apply`) instead.  The
switch is read once per process, so the second family runs in a child process.  Both are
checked against the FP64 oracle (L1 <= 1e-9 per (rate set, x0)) and against each other
(L1 <= 1e-9) on an n=16 network whose largest level groups hold 8,852 states.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
from paraexastolog_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import paraexastolog_b200 as esl
from paraexastolog_b200 import synth
net_g = synth.precision_network(seed=1, n=16)
rates = synth.log_uniform_rates(np.random.default_rng(1), 16, 64)
x0 = synth.dirichlet_subspace_x0(np.random.default_rng(2), 16, np.arange(6))
ctx = esl.Context(0)
net = esl.Net.build(ctx, esl.Model.parse(net_g.bnet), rates[0])
res = esl.solve_batch(ctx, net, rates, x0[None], method=esl.METHOD_DIRECT)
assert res.report.converged == 1
np.save(sys.argv[2], res.x_inf[:, 0].cpu().numpy())
"""


@pytest.fixture(scope="module")
def esl():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import paraexastolog_b200 as E
    E.lib()
    return E


def _solve_in_child(tmp_path, op):
    out = tmp_path / f"xinf_{op}.npy"
    env = dict(os.environ, ESL_SWEEP_OP=op)
    subprocess.run([sys.executable, "-c", CHILD, REPO, str(out)], env=env, check=True, timeout=600)
    return np.load(out)


def test_paired_and_per_lane_operators_agree(esl, tmp_path):
    paired = _solve_in_child(tmp_path, "paired")
    per_lane = _solve_in_child(tmp_path, "reg")
    assert np.abs(paired - per_lane).sum(1).max() <= 1e-9
    net_g = synth.precision_network(seed=1, n=16)
    rates = synth.log_uniform_rates(np.random.default_rng(1), 16, 64)
    x0 = synth.dirichlet_subspace_x0(np.random.default_rng(2), 16, np.arange(6))
    sym = O.Model(text=net_g.bnet).analyse(rates[0])
    for b in (0, 31, 63):
        ox, _ = sym.solve(x0, rates[b])
        assert np.abs(paired[b] - ox).sum() <= 1e-9, b
        assert np.abs(per_lane[b] - ox).sum() <= 1e-9, b
