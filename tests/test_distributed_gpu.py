"""Gram sharding (sigpde_b200.distributed) with the CUDA engine on one GPU.

Only one GPU is available to a test here, and NCCL puts at most one rank on a
device, so the ranks are simulated: every rank's row block (rank_rows, with the
engine's own solve hooks: a Gram left of the diagonal block, a symmetric Gram
on it) is computed in turn on cuda:0 and stacked, which is what the all-gather
assembles (its host logic is tested with gloo ranks in test_distributed_cpu).
The result must equal the single-call Gram: bitwise for a Gram, within 1e-12
relative for a symmetric Gram (its off-diagonal blocks come from the Gram
kernels, the single call takes the symmetric kernel), and exactly symmetric.
The process-group-free call (world 1) is the single-call Gram itself.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [1, 2, 4])
def test_simulated_ranks_equal_the_single_gram(world, oracle):
    import sigpde_b200.torch as sig
    from sigpde_b200 import distributed as D
    x = torch.tensor(oracle.brownian(37, 40, 6, 81), dtype=torch.float64, device="cuda")
    y = torch.tensor(oracle.brownian(29, 33, 6, 82), dtype=torch.float64, device="cuda")
    sx = torch.linspace(0.7, 1.3, 37, dtype=torch.float64, device="cuda")
    k = sig.SigPDE(sig.kernels.LinearKernel(), 1)
    solve = D._engine_gram(sig.kernels.LinearKernel(), 1, "fp64")
    for yy, s in ((y, None), (None, None), (None, sx)):
        rows = [D.rank_rows(x, yy, s, None, r, world, solve)[1] for r in range(world)]
        got = D.assemble(torch.cat(rows, 0), yy is None).cpu().numpy()
        want = k.gram(x, yy, s, None).cpu().numpy()
        if yy is not None:
            np.testing.assert_array_equal(got, want)
        else:
            np.testing.assert_array_equal(got, got.T)
            assert float(np.max(np.abs(got - want) / np.abs(want))) <= 1e-12
    assert torch.equal(D.sharded_gram(x, y, dyadic_order=1), k.gram(x, y))


def test_robust_without_a_process_group(oracle):
    import sigpde_b200.torch as sig
    from sigpde_b200 import distributed as D
    rng = np.random.default_rng(8)
    x = torch.tensor(oracle.brownian(24, 30, 5, 83, scale=np.exp(rng.uniform(np.log(0.5), np.log(4.0), 24))),
                     dtype=torch.float64, device="cuda")
    got = D.sharded_robust_gram(x, dyadic_order=1).cpu().numpy()
    want = sig.RobustSigPDE(sig.kernels.LinearKernel(), 1).gram(x).cpu().numpy()
    np.testing.assert_array_equal(got, got.T)
    assert float(np.max(np.abs(got - want) / np.abs(want))) <= 1e-12
