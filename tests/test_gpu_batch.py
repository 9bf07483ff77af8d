"""Many networks in one call (esl_solve_many): uneven random networks, several rate sets
and initial distributions each, run concurrently over a pool of contexts.  Every
result matches the same job solved alone (L1 <= 1e-12 in FP64; 1e-10 for the mixed
method, whose FP32 reductions run in a different order) and the FP64 oracle
(L1 <= 1e-9)."""
import numpy as np
import pytest

import oracle as O
from paraexastolog_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def esl():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import paraexastolog_b200 as E
    E.lib()
    return E


def _jobs(esl, ctxs, count=6, seed=11):
    rng = np.random.default_rng(seed)
    jobs, specs = [], []
    for i in range(count):
        n = int(rng.integers(9, 13))
        g = synth.random_table_network(rng, n, [3], 0.5)
        rates = synth.log_uniform_rates(rng, n, 4)
        xs = np.stack([synth.dirichlet_subspace_x0(rng, n, rng.choice(n, 4, replace=False)) for _ in range(3)])
        net = esl.Net.build(ctxs[i % len(ctxs)], esl.Model.parse(g.bnet), rates[0])
        jobs.append((net, rates, xs))
        specs.append((g.bnet, rates, xs))
    return jobs, specs


@pytest.mark.parametrize("method", ["direct", "mixed"])
def test_solve_many_matches_single_and_oracle(esl, method):
    m = {"direct": esl.METHOD_DIRECT, "mixed": esl.METHOD_MIXED}[method]
    ctxs = [esl.Context(0, torch.cuda.Stream()) for _ in range(3)]
    jobs, specs = _jobs(esl, ctxs)
    res = esl.solve_many(ctxs, jobs, method=m, tol=1e-11)
    for (net, rates, xs), (text, _, _), r in zip(jobs, specs, res):
        assert r.report.converged == 1
        alone = esl.solve_batch(ctxs[0], net, rates, xs, method=m, tol=1e-11)
        torch.cuda.synchronize()
        a, b = r.x_inf.cpu().numpy(), alone.x_inf.cpu().numpy()
        assert np.abs(a - b).sum(-1).max() <= (1e-12 if method == "direct" else 1e-10)
        sym = O.Model(text=text).analyse(rates[0])
        for k in (0, 3):
            for q in (0, 2):
                ox, om = sym.solve(xs[q], rates[k])
                assert np.abs(a[k, q] - ox).sum() <= 1e-9
                assert np.abs(r.marginals[k, q].cpu().numpy() - om).max() <= 1e-9


def test_solve_many_reports_a_failing_job(esl):
    ctxs = [esl.Context(0, torch.cuda.Stream()) for _ in range(2)]
    jobs, _ = _jobs(esl, ctxs, count=3, seed=5)
    net, rates, xs = jobs[1]
    bad = rates.copy()
    bad[:, 0] = 0.0  # a zero pattern the net was not built for
    jobs[1] = (net, bad, xs)
    with pytest.raises(esl.EslError):
        esl.solve_many(ctxs, jobs, method=esl.METHOD_DIRECT)


def test_many_network_workload_full_size(esl):
    """The many-network workload at its stated size: 48 random networks (n = 12..18,
    uneven), 64 rate sets x 16 initial distributions each, 49,152 solves in one
    esl_solve_many call over four contexts.  Every job converges; two seeded (rate set,
    x0) pairs per network are checked against the FP64 oracle (L1 <= 1e-9)."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    w = synth.config_batch()
    ctxs = [esl.Context(0, torch.cuda.Stream()) for _ in range(4)]
    jobs = []
    for i, (net_g, rates, xs) in enumerate(zip(w.networks, w.rates, w.x0)):
        net = esl.Net.build(ctxs[i % len(ctxs)], esl.Model.parse(net_g.bnet), rates[0])
        jobs.append((net, rates, xs))
    res = esl.solve_many(ctxs, jobs, method=esl.METHOD_DIRECT, tol=1e-10)
    assert sum(r.x_inf.shape[0] * r.x_inf.shape[1] for r in res) == 48 * 64 * 16
    assert all(r.report.converged == 1 and r.status == 0 for r in res)
    rng = np.random.default_rng(48)
    picks = [(rng.integers(0, 64, 2), rng.integers(0, 16, 2)) for _ in range(48)]

    def oracle_job(i):
        net_g, rates, xs = w.networks[i], w.rates[i], w.x0[i]
        kb, kq = picks[i]
        sym = O.Model(text=net_g.bnet).analyse(rates[0])
        return sym.solve_many(rates[kb], xs[kq], threads=1)

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        refs = list(ex.map(oracle_job, range(48)))
    for i, (r, (ox, om)) in enumerate(zip(res, refs)):
        kb, kq = picks[i]
        got = r.x_inf[torch.as_tensor(kb), torch.as_tensor(kq)].cpu().numpy()
        gm = r.marginals[torch.as_tensor(kb), torch.as_tensor(kq)].cpu().numpy()
        assert np.abs(got - ox).sum(1).max() <= 1e-9, i
        np.testing.assert_allclose(gm, om, atol=1e-9, rtol=0)
