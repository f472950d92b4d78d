"""Failures injected on the host, none of which faults, traps or hangs the
GPU: a non-finite value in a right-hand side, an iteration budget of one,
and a zero right-hand side, for the batched, assembled and nonlinear solves.
Every solve returns, and reports the failure in its status and diagnostics
(per problem for a batch) while the other problems of the batch finish.
The TMA Laplacian's pipeline waits are given a bound of zero polls, so they
run out: the kernel stops, lets its loads in flight land and returns, the
plan reports SIL_ERR_BUDGET and the context stays usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIL_OK, SIL_ERR_NONFINITE = 0, 5
SIL_ERR_BUDGET = 7


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_batched_solve_reports_a_nonfinite_problem_and_finishes_the_others(torch):
    import similie_b200.magnetostatics as mag
    from similie_b200 import _native
    rng = np.random.default_rng(41)
    probs = [mag.synthetic_problem(rng, n, cores=1) for n in (33, 49)]
    rhs0 = probs[0].rhs()
    rhs0[16 + 33 * 16] = np.nan
    mus = [_dev(torch, p.node_mu()) for p in probs]
    rhss = [_dev(torch, rhs0), _dev(torch, probs[1].rhs())]
    sols = [torch.zeros_like(r) for r in rhss]
    arr = (_native.SilMag2dProblem * 2)()
    for k, (p, n) in enumerate(zip(probs, (33, 49))):
        arr[k].nx = arr[k].ny = n
        arr[k].node_mu = mus[k].data_ptr()
        arr[k].rhs = rhss[k].data_ptr()
        arr[k].solution = sols[k].data_ptr()
    st = _native.SilSolveSettings()
    st.max_iterations = 20000
    st.relative_tolerance = 1e-10
    diag = (_native.SilSolveDiagnostics * 2)()
    rc = _native.lib().sil_mag2d_solve_batch(arr, 2, ctypes.byref(st), diag,
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == SIL_ERR_NONFINITE
    assert diag[0].status == SIL_ERR_NONFINITE and not diag[0].converged
    assert diag[1].status == SIL_OK and diag[1].converged


def test_iteration_budget_of_one(torch):
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(42)
    p = mag.synthetic_problem(rng, 33, cores=1)
    rhs = _dev(torch, p.rhs())
    x = torch.zeros_like(rhs)
    d = mag.solve_batch([_dev(torch, p.node_mu())], [rhs], [x], [(33, 33)], solver="cg", max_iterations=1)
    assert not d[0].converged and d[0].iterations <= 1 and d[0].status == SIL_OK


def test_assembled_solve_reports_nonfinite_and_budget(torch):
    import similie_b200.assembled as asm
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(43)
    p = mag.synthetic_problem(rng, 33, cores=1)
    A = asm.CsrMatrix.mag2d(33, 33, _dev(torch, p.node_mu()))
    P = asm.Preconditioner(A, "jacobi")
    rhs = p.rhs()
    x = torch.zeros(33 * 33, dtype=torch.float64, device="cuda")
    d = asm.solve(A, P, _dev(torch, rhs), x, max_iterations=1)
    assert not d.converged and d.iterations == 1 and d.status == SIL_OK
    bad = rhs.copy()
    bad[16 + 33 * 16] = np.inf
    d = asm.solve(A, P, _dev(torch, bad), x)
    assert d.status == SIL_ERR_NONFINITE and not d.converged


def test_nonlinear_solve_reports_nonfinite(torch):
    import similie_b200.magnetostatics as mag
    p, mu, fe, b, h = mag.nonlinear_problem(33, 3)
    rhs = p.rhs()
    rhs[16 + 33 * 16] = np.nan
    x = torch.zeros(33 * 33, dtype=torch.float64, device="cuda")
    d = mag.nl_solve_batch([_dev(torch, mu)], [_dev(torch, fe)], [(b, h)], [_dev(torch, rhs)], [x], [(33, 33)])
    assert d[0].status == SIL_ERR_NONFINITE and not d[0].converged and d[0].refinements == 0


def test_laplacian_wait_that_runs_out_reports_budget(torch):
    import oracle as O
    import similie_b200 as sil
    from helpers import gaussian_random_field, rel_err
    n = 512
    w = gaussian_random_field(n, seed=5)
    coords = [np.arange(n) / n, np.arange(n) / n]
    geo = sil.Geometry(coords)
    inp = torch.from_numpy(w).cuda()
    out = torch.zeros((n - 1, n - 1, 2), dtype=torch.float64, device="cuda")
    bad = sil.make_staged_laplacian(geo, out, inp, 1)
    assert bad.kernel == 2
    bad.run(out, inp)           # first run: the pipeline shape is tuned with the default bound
    bad.status()
    bad.set_wait_bound(0)
    bad.run(out, inp)
    with pytest.raises(sil.SilError) as e:
        bad.status()
    assert e.value.status == SIL_ERR_BUDGET
    # the context is still usable: a fresh plan computes the right Laplacian
    good = sil.make_staged_laplacian(geo, out, inp, 1)
    good.run(out, inp)
    good.status()
    ref = O.laplacian(2, 1, O.position_from_coords(coords), w)
    assert rel_err(out.cpu().numpy(), ref) <= 1e-12
