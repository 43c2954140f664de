"""What the trained workload estimator gains (GPU).

The learned scheduler's network (sjoin/estimator_c4.bin, trained by the
engine's own kernels on seeded runs of the 6-D exponential generator) predicts
per-cell pair counts from cell features, which size the result batches and
order the work queue.  The method without it is either the sampling estimate
(every 100th point counts its neighbours first) or the same network untrained.
On a 6-D exponential set the trained network must
  * leave the pair set unchanged (it only schedules),
  * predict the pair total within a factor of two, where an untrained network
    is off by orders of magnitude and makes the join several times slower,
  * replace the sampling pass (a fraction of its time) while planning about
    as many batches.
"""
import os

import pytest

import sjoin

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(sjoin.__file__), "estimator_c4.bin")


def _run(pts, eps, which):
    kw = dict(mode=10, precision=sjoin.PREC_FP32_REFINE, capacity=100_000_000)
    if which != "sampling":
        kw["scheduler"] = sjoin.SCHED_LEARNED
    with sjoin.SelfJoin(6, eps, **kw) as sj:
        if which == "trained":
            sj.load_estimator(WEIGHTS)
        elif which == "untrained":
            sj.set_estimator(sjoin.mlp_init(3))
        sj.set_points(pts)
        sj.build_index()
        sj.join(sjoin.DELIVER_NONE)          # warm-up (allocations)
        sj.build_index()
        return sj.join(sjoin.DELIVER_NONE)


def test_trained_estimator_gain():
    pts = sjoin.datasets.exponential(300_000, 6, 40.0, 4343)
    eps = 0.03
    st = {w: _run(pts, eps, w) for w in ("sampling", "trained", "untrained")}
    meas = st["sampling"].total_pairs
    for w in st:
        assert st[w].total_pairs == meas and st[w].pair_hash == st["sampling"].pair_hash, w
    ratio_trained = st["trained"].estimated_pairs / meas
    ratio_untrained = st["untrained"].estimated_pairs / meas
    assert 0.5 < ratio_trained < 2.0, ratio_trained
    assert ratio_untrained < 0.01, ratio_untrained
    assert st["trained"].ms_estimate < 0.25 * st["sampling"].ms_estimate
    assert st["trained"].num_batches <= 1.5 * st["sampling"].num_batches
    assert st["trained"].ms_total < 0.5 * st["untrained"].ms_total
