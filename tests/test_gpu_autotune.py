"""GPU: the batch autotuner.

A quick tuning run (tile size per class, then threads per CTA jointly with
CTAs per SM on a mixed batch) writes a table that loads into Batch and leaves
every output byte unchanged against the shipped table; every CTA size the
kernel takes gives the same bytes, and an unsupported one is refused.
"""

import json

import pytest

from quicktex_b200 import autotune, capi
from quicktex_b200.batch import Batch, load_tuning, run_jobs

from .test_gpu_batch import make_jobs

pytestmark = pytest.mark.gpu


def test_quick_tuning_table_loads_and_keeps_outputs(tmp_path):
    table = autotune.tune(0, quick=True)
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps(table))
    tuned = load_tuning(str(path))
    assert tuned["threads_per_cta"] in autotune.THREADS
    assert tuned["ctas_per_sm"] * tuned["threads_per_cta"] <= 16 * 32
    assert {(r["format"], r["level"]) for r in tuned["rules"] if r["op"] == 0 and r["format"] in (1, 3)} == \
        {(f, L) for f in (1, 3) for L in range(20)}
    jobs, _ = make_jobs(21, 60)
    shipped = run_jobs(jobs)
    b = Batch(0, tuning=tuned)
    try:
        assert run_jobs(jobs, batch=b) == shipped
    finally:
        b.close()


@pytest.mark.parametrize("threads", [32, 64, 128])
def test_every_cta_size_gives_the_same_bytes(threads):
    jobs, _ = make_jobs(22, 40)
    ref = run_jobs(jobs)
    b = Batch(0)
    try:
        b.set_threads(threads)
        b.set_grid(0)
        assert run_jobs(jobs, batch=b) == ref
    finally:
        b.close()


def test_unsupported_cta_size_is_refused():
    b = Batch(0)
    try:
        with pytest.raises(capi.QtError):
            b.set_threads(48)
    finally:
        b.close()
