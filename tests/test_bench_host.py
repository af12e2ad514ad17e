"""The bench's host logic on the CPU: its defaults, the flop and byte models behind `roofline`, the
measured-traffic scaling, the shape replay of the end-to-end leg and the CPU-baseline row sizing."""

import argparse

import numpy as np
import pytest

import bench
from grasph2_b200.params import config0_params, config1_params, config2_params


def test_defaults_are_the_headline_workload():
    a = bench.parse([])
    assert a.gpus == 1 and a.impl == "ours"
    assert a.workload == "plummer" and a.n == 0      # N = 2^20 Plummer sphere
    assert a.warmup >= 3 and a.steps >= 1            # at least three untimed warm-up steps
    assert a.legs == "auto"


def test_flop_model_per_workload():
    n = 1000
    st = {"mass": np.zeros(n)}
    grav = bench.flops_per_step(config2_params(), st, 0, culled=True)
    assert grav == {"gravity": bench.FLOP_GRAV_PAIR * n * n}   # 20 flop per ordered pair
    nb = 12345
    culled = bench.flops_per_step(config1_params(), st, nb, culled=True)
    assert culled["gravity"] == bench.FLOP_GRAV_PAIR * n * n
    assert culled["density"] == bench.FLOP_DENS_NB * nb     # culled: only neighbour work in the SPH slots
    assert culled["pairs"] == bench.FLOP_FUSED_NB * nb      # solids: the fused per-neighbour count
    allp = bench.flops_per_step(config1_params(), st, nb, culled=False)
    assert allp["density"] == bench.FLOP_DENS_NB * nb + bench.FLOP_DENS_PAIR * n * n
    assert allp["pairs"] == bench.FLOP_FUSED_NB * nb + bench.FLOP_GRAV_PAIR * n * n
    fluid = bench.flops_per_step(config0_params(), st, nb, culled=True)
    assert fluid["pairs"] == bench.FLOP_ACC_NB * nb


def test_integrator_bytes_match_the_survey_model():
    assert bench.integrator_bytes(config1_params()) == 196   # impact: SPH + solids
    assert bench.integrator_bytes(config2_params()) == 112   # gravity alone
    assert bench.integrator_bytes(config0_params()) == 124   # fluid SPH


def test_measured_traffic_scales_with_particles():
    key = ("plummer", "gravity", "symmetric", 128)
    b, n = bench.MEASURED_TRAFFIC[key]
    # the captured case is smaller than the headline; the line reports bytes per particle x N
    assert n < (1 << 20)
    assert b * (1 << 20) / n == pytest.approx(4 * b)
    for (workload, kernel, form, g), (bytes_, parts) in bench.MEASURED_TRAFFIC.items():
        assert bytes_ > 16 * parts      # at least the j-records once
        assert form in ("symmetric", "one-sided")


def test_shape_options_replay_the_tuned_gravity_shape():
    sym = bench.shape_options({"grav_sym_groups": 128}, {"accum": "plain"})
    assert sym == {"accum": "plain", "gravity": "symmetric", "gravity_groups": 128}
    one = bench.shape_options({"grav_sym_groups": 0, "grav_ipt": 4, "grav_jt": 256, "grav_nseg": 8}, {})
    assert one == {"gravity": "one-sided", "i_per_thread": 4, "j_tile": 256, "j_split": 8}


def test_leg_args_copy_and_override():
    a = bench.parse([])
    b = bench.leg_args(a, workload="impact", steps=300)
    assert b.workload == "impact" and b.steps == 300
    assert a.workload == "plummer" and a.steps != 300   # the headline's arguments are untouched
    assert isinstance(b, argparse.Namespace)


def test_rows_for_budget_grows_to_the_budget_and_stops_at_n():
    calls = []

    def sample(m):  # 1 ms per row
        calls.append(m)
        return (1e-3 * m,)
    m = bench.rows_for_budget(sample, 1 << 20, 2.0)
    assert 1000 <= m <= 4000 and calls[0] == 64
    m_small = bench.rows_for_budget(sample, 300, 100.0)
    assert m_small == 300                               # never more rows than particles


def test_whole_job_rate_counts_every_rank():
    assert bench.whole_job_rate(20, 4, 1000.0) == pytest.approx(80.0)
    assert bench.max_over_ranks(3.5) == 3.5
