"""The batched and served forms: many placements at once on one GPU.

A job is exactly one GlobalPlacer.run; running it in a mix with others must not
change its result, in either server mode: batched (the running jobs'
evaluations share one launch per kernel family and round, and every block of a
batched launch does what the same block of the job's own launch does) or
concurrent (every job launches its own kernels).  Admission must respect the
memory budget.
"""
from __future__ import annotations

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from myplacement_b200.design import small_instance


def _job(cells: int, seed: int, iterations: int = 60):
    design, bins = small_instance(cells, seed)
    x, y = mp.random_placement(design, seed)
    design = design.copy_with_positions(x, y)
    options = mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9, iterations=iterations)
    return design, options


def test_footprint_estimate_grows_with_the_design():
    small = _job(1000, 1)
    large = _job(4000, 2)
    a = mp.estimate_bytes(*small)
    b = mp.estimate_bytes(*large)
    assert 0 < a < b


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_served_results_equal_alone(gpu, batched):
    """Three jobs give bit-identical placements alone and inside a mix of eight."""
    probes = [_job(2000, 11), _job(3500, 12), _job(1200, 13)]
    alone = [mp.GlobalPlacer().run(d, o) for d, o in probes]
    fillers = [_job(cells, 20 + k) for k, cells in enumerate((3000, 1500, 2500, 4000, 1800))]
    order = [fillers[0], probes[0], fillers[1], fillers[2], probes[1], fillers[3], probes[2], fillers[4]]
    with mp.PlacementServer(device=0, workers=4, batched=batched) as server:
        ids = [server.submit(d, o) for d, o in order]
        results = []
        for job in ids:
            assert server.wait(job, 300.0)
            results.append(server.take(job))
        stats = server.stats()
    assert stats["completed"] == 8 and stats["failed"] == 0
    assert stats["peak_running"] >= 2  # the jobs did overlap on the device
    assert stats["batched"] == int(batched)
    if batched:  # iterations of several jobs went into shared launches
        assert stats["batch_rounds"] > 0 and stats["batch_peak_round"] >= 2
        assert stats["batch_evaluations"] > stats["batch_rounds"]
    mixed = [results[1], results[4], results[6]]
    for (placed, job_stats), reference in zip(mixed, alone):
        np.testing.assert_array_equal(placed.module_x, reference.module_x)
        np.testing.assert_array_equal(placed.module_y, reference.module_y)
        assert placed.hpwl_after == reference.hpwl_after
        assert placed.completed_iterations == reference.completed_iterations
        assert len(placed.history) == len(reference.history)
        assert job_stats["reserved_bytes"] <= job_stats["estimated_bytes"]
        assert job_stats["latency_seconds"] >= job_stats["run_seconds"] > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_batch_place_matches_global_place(gpu, batched):
    """Instances of uneven sizes and bin grids (32 x 32 to 128 x 128 bins: contractions of
    one and of two K splits in one round) match their plain runs bit for bit.  A plain
    run launches the momentum lookahead behind the current evaluation and hands the
    accepted step's velocity update and checkpoint copy to the next gather; a batched
    instance takes one evaluation at a time, so equal results also show that the
    overlap changes nothing."""
    jobs = [_job(cells, 40 + k, iterations=40) for k, cells in enumerate((1000, 2600, 1700, 3100, 1300, 2200, 9000))]
    placed, job_stats, server_stats = mp.batch_place([d for d, _ in jobs], [o for _, o in jobs], workers=4,
                                                     batched=batched)
    assert server_stats["completed"] == len(jobs)
    for (design, options), result in zip(jobs, placed):
        reference = mp.GlobalPlacer().run(design, options)
        np.testing.assert_array_equal(result.module_x, reference.module_x)
        np.testing.assert_array_equal(result.module_y, reference.module_y)
        assert result.hpwl_after == reference.hpwl_after


@pytest.mark.gpu
def test_admission_respects_the_memory_budget(gpu):
    jobs = [_job(1500, 60 + k, iterations=20) for k in range(3)]
    largest = max(mp.estimate_bytes(d, o) for d, o in jobs)
    # Room for one job at a time: they must run one after another.
    with mp.PlacementServer(device=0, workers=3, memory_budget=int(largest * 1.5)) as server:
        ids = [server.submit(d, o) for d, o in jobs]
        for job in ids:
            assert server.wait(job, 300.0)
            server.take(job, history=False)
        stats = server.stats()
        assert stats["peak_running"] == 1
        assert stats["peak_reserved"] <= stats["memory_budget"]
        # A job that cannot fit even alone is refused at submission.
        big, big_options = _job(20000, 70)
        with pytest.raises(mp.EngineError) as error:
            server.submit(big, big_options)
        assert error.value.status == _abi.MPGP_ERR_BUDGET


def test_server_needs_a_gpu():
    from conftest import GPU_PRESENT

    if GPU_PRESENT:
        pytest.skip("a GPU is present")
    with pytest.raises(mp.EngineError):
        mp.PlacementServer(device=0, workers=2)


@pytest.mark.gpu
@pytest.mark.parametrize("solve", ["default", "banded"])
def test_batched_banded_field_solve_matches_plain(gpu, monkeypatch, solve):
    """Grids taller than 256 rows take the banded field solve: in a batched round one
    launch per cluster shape, and inverse-only launches for the evaluations that reuse
    the last density.  With MPGP_FIELD_SOLVE=banded the small grids take it too (clusters
    of four and eight CTAs of 16 columns).  Batched results equal the plain runs."""
    if solve == "banded":
        monkeypatch.setenv("MPGP_FIELD_SOLVE", "banded")
    else:
        monkeypatch.delenv("MPGP_FIELD_SOLVE", raising=False)
    jobs = []
    for cells, bins, seed in ((2500, 320, 81), (1800, 448, 82), (1200, 64, 83), (3000, 128, 84), (2200, 256, 85)):
        design, _ = small_instance(cells, seed)
        x, y = mp.random_placement(design, seed)
        design = design.copy_with_positions(x, y)
        jobs.append((design, mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9, iterations=30)))
    placed, _, server_stats = mp.batch_place([d for d, _ in jobs], [o for _, o in jobs], workers=5, batched=True)
    assert server_stats["completed"] == len(jobs)
    for (design, options), result in zip(jobs, placed):
        reference = mp.GlobalPlacer().run(design, options)
        np.testing.assert_array_equal(result.module_x, reference.module_x)
        np.testing.assert_array_equal(result.module_y, reference.module_y)
        assert result.hpwl_after == reference.hpwl_after
