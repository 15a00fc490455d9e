"""Host logic of the batch runner (no device work): formulations, the
concurrency policy by problem size and the per-problem memory model that
sizes the waves."""
import pytest

from neuralat_b200.bem.batch import FORMULATIONS, BatchRunner, problem_bytes


def test_formulations_and_validation():
    assert FORMULATIONS == ("cbie", "burton_miller")
    with pytest.raises(ValueError):
        BatchRunner(memory_budget_bytes=1 << 30, formulation="hbie-typo")


def test_concurrency_follows_problem_size():
    with BatchRunner(memory_budget_bytes=1 << 30, workers=4) as r:
        assert r.concurrency(162) == 4
        assert r.concurrency(2562) == 4
        assert r.concurrency(10242) == 2  # one such solve already keeps every SM busy
    with BatchRunner(memory_budget_bytes=1 << 30, workers=1) as r:
        assert r.concurrency(10242) == 1 and r.concurrency(162) == 1


def test_problem_bytes_counts_matrices_and_krylov_basis():
    n, m, R = 1000, 8, 200
    b = problem_bytes(n, m, R)
    assert b >= 3 * 8 * n * n  # V, the left-hand side and the tensor-core planes
    assert b >= 8 * m * (R + 1) * n  # the complex64 Krylov basis
    ratio = problem_bytes(2 * n, m, R) / b  # dense matrices quadratic, basis linear in n
    assert 2.0 < ratio <= 4.0
    assert problem_bytes(n, 2 * m, R) > b


def test_plan_waves_groups_by_class_and_budget():
    from neuralat_b200.bem.batch import plan_waves

    def conc(nv):
        return 2 if nv >= 4096 else 4

    sizes = [("a", 10242, 40), ("b", 10242, 40), ("c", 10242, 40), ("d", 642, 5), ("e", 642, 5)]
    waves = plan_waves(sizes, budget=100, concurrency=conc)
    assert waves == [(["a", "b"], 2), (["c"], 2), (["d", "e"], 4)]
    assert all(sum(b for j, _, b in sizes if j in w) <= 100 for w, _ in waves)


def test_plan_waves_refuses_a_problem_above_the_budget():
    from neuralat_b200.bem.batch import plan_waves

    with pytest.raises(MemoryError):
        plan_waves([("a", 642, 5), ("b", 10242, 101)], budget=100, concurrency=lambda nv: 1)
    with pytest.raises(ValueError):
        BatchRunner(memory_budget_bytes=0)
