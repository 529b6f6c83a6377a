"""The self-join plan (head width p, rare-feature threshold C) computed on
the host by cuapss_plan_self_join: no device needed. The GPU run makes the
same choice (tests/test_gpu_rare.py checks the two agree); the benchmark
lines record the run's choice (n = d = 1M: p = 1,024, C = 1,024,
3,167,300,348 explicit pairs; its 200,000-row prefix: p = 960, C = 256,
163,951,608 pairs)."""
import numpy as np
import pytest

import cuapss
from cuapss import synth


@pytest.fixture(scope="module")
def zipf200k():
    return synth.generate("mixed_1m", n=200_000)


def test_plan_of_the_200k_prefix(zipf200k):
    plan = cuapss.plan_self_join(zipf200k)
    assert plan == {"head_width": 960, "rare_max_count": 256, "explicit_pairs": 163_951_608}


def test_plan_of_the_headline_workload():
    x = synth.generate("mixed_1m")
    plan = cuapss.plan_self_join(x)
    assert plan == {"head_width": 1024, "rare_max_count": 1024,
                    "explicit_pairs": 3_167_300_348}


def test_pairs_bound_and_precision(zipf200k):
    full = cuapss.plan_self_join(zipf200k)
    for bound in (10**8, 10**7, 10**6):
        p = cuapss.plan_self_join(zipf200k, max_pairs=bound)
        assert p["explicit_pairs"] <= bound
        assert p["rare_max_count"] <= full["rare_max_count"]
        assert p["head_width"] % 64 == 0
    # a smaller pair budget leaves more tail to probe, so the head widens
    assert cuapss.plan_self_join(zipf200k, max_pairs=10**6)["head_width"] >= full["head_width"]
    fp32 = cuapss.plan_self_join(zipf200k, cuapss.PREC_FP32)
    assert fp32["head_width"] == 64 and fp32["rare_max_count"] > 0


def test_small_joins_plan_no_pairs():
    x = synth.generate("mixed_1m", n=20_000)
    plan = cuapss.plan_self_join(x)
    assert plan["rare_max_count"] == 0 and plan["explicit_pairs"] == 0


def test_counts_form_and_thresholds():
    rng = np.random.default_rng(3)
    d, n = 50_000, 100_000
    counts = np.minimum(rng.zipf(1.3, size=d), n).astype(np.int32)
    plan = cuapss.plan_self_join((counts, n))
    c = plan["rare_max_count"]
    assert c in (0, 16, 32, 64, 128, 256, 512, 1024, 2048)
    if c:
        sel = counts[counts <= c].astype(np.int64)
        assert plan["explicit_pairs"] == int((sel * (sel - 1) // 2).sum())
    # a feature in no row, and one in every row, are valid counts
    counts[0], counts[1] = 0, n
    cuapss.plan_self_join((counts, n))


def test_bad_arguments():
    counts = np.array([1, 2, 3], np.int32)
    with pytest.raises(cuapss.CuapssError):
        cuapss.plan_self_join((counts, 2))  # a count above n
    with pytest.raises(cuapss.CuapssError):
        cuapss.plan_self_join((counts, 10), precision=7)
    with pytest.raises(cuapss.CuapssError):
        cuapss.plan_self_join((np.array([-1], np.int32), 10))
