"""Host logic of the benchmark workloads and the request loop (no GPU)."""

import numpy as np

from foilbench_b200 import workloads


def test_batched_mix_is_seeded_and_within_the_stated_ranges():
    a = workloads.batched_mix(11, 64)
    b = workloads.batched_mix(11, 64)
    assert [s.id for s in a] == [s.id for s in b]
    for sc in a:
        assert (sc.domain.nx, sc.domain.ny) in workloads.GRID_CHOICES
        code = sc.foil.naca
        assert 0 <= int(code[0]) <= 4 and 9 <= int(code[2:]) <= 18
        assert -5.0 <= sc.control_at(0.0).angle_degrees <= 20.0
        assert 100.0 <= sc.reynolds <= 1.0e4
        assert sc.precision == "float32"
        assert abs(sc.output_dt - 0.5 * min(4.0 / sc.domain.nx, 2.0 / sc.domain.ny)) < 1e-15
        # every drawn grid qualifies for batched launches (nx multiple of 16, 129..2048)
        assert sc.domain.nx % 16 == 0 and 129 <= sc.domain.nx <= 2048


def test_request_stream_is_poisson_like():
    reqs = workloads.request_stream(3, rate_per_s=200.0, duration_s=20.0)
    t = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 20.0
    assert abs(len(reqs) / 20.0 - 200.0) < 25.0
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 2000
