"""The batched form (many independent samples in one persistent, graph-captured
launch) against the oracle, sample by sample: FP64 within 1e-9 A, FP32C within
the compensated form's 2e-5 A; the resident plan replays its graph."""
import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import backend as B
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _small_batch(seed=9, n=10):
    return W.batch(nsamples=n, edge=(5, 11), nloops=(1, 5), radius=(4.0, 9.0), segments=(16, 40),
                   images=(1, 2), seed=seed)


@pytest.mark.parametrize("split", [1, 2, 4, 8])
def test_batch_fp64_matches_oracle(split):
    batch = _small_batch()
    us, _ = B.batch_gpu(batch, C.DISCO_FP64, image_split=split)
    for w, u in zip(batch, us):
        ref = O.displace(w.x, w.y, w.z, w.loops, w.box, images=w.images, nu=w.nu)
        assert max(np.abs(u[k] - ref[k]).max() for k in range(3)) <= 1e-9, w.name


@pytest.mark.parametrize("stage_kb", [16, 24, 48])
def test_batch_fp32c_matches_oracle(stage_kb):
    batch = _small_batch(seed=10)
    us, _ = B.batch_gpu(batch, C.DISCO_FP32C, stage_kb=stage_kb)
    for w, u in zip(batch, us):
        ref = O.displace(w.x, w.y, w.z, w.loops, w.box, images=w.images, nu=w.nu)
        assert max(np.abs(u[k] - ref[k]).max() for k in range(3)) <= 2e-5, w.name


def test_batch_many_chunks_and_empty_samples():
    """A sample whose table spans several 16 KB stages, a sample without loops
    and a sample without atoms, in the same batch."""
    batch = _small_batch(seed=11, n=4)
    big = W.batch(nsamples=1, edge=(6, 6), nloops=(12, 12), radius=(8.0, 9.0), segments=(120, 128),
                  images=(1, 1), seed=12)[0]
    noloops = W.Workload("noloops", batch[0].x, batch[0].y, batch[0].z, [], batch[0].box, 1, 0.29, "line")
    noatoms = W.Workload("noatoms", np.zeros(0), np.zeros(0), np.zeros(0), batch[1].loops, batch[1].box,
                         1, 0.29, "line")
    allw = batch + [big, noloops, noatoms]
    us, _ = B.batch_gpu(allw, C.DISCO_FP64, stage_kb=16)
    for w, u in zip(allw, us):
        if w.n == 0:
            continue
        ref = O.displace(w.x, w.y, w.z, w.loops, w.box, images=w.images, nu=w.nu)
        assert max(np.abs(u[k] - ref[k]).max() for k in range(3)) <= 1e-9, w.name


def test_batch_plan_graph_replay_accumulates():
    torch = pytest.importorskip("torch")
    batch = _small_batch(seed=13, n=6)
    pos = [torch.tensor(np.stack([w.x, w.y, w.z]), dtype=torch.float64, device="cuda") for w in batch]
    u = [torch.zeros_like(p) for p in pos]
    ptrs = [(p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(), q[0].data_ptr(), q[1].data_ptr(),
             q[2].data_ptr()) for p, q in zip(pos, u)]
    plan = B.BatchPlan(batch, ptrs, precision=C.DISCO_FP64)
    plan.execute()
    plan.execute()
    plan.sync()
    for w, q in zip(batch, u):
        ref = np.stack(O.displace(w.x, w.y, w.z, w.loops, w.box, images=w.images, nu=w.nu))
        assert np.abs(q.cpu().numpy() - 2 * ref).max() <= 2e-9
    st = plan.stats()
    assert st["evals_per_atom"] == sum(w.n * w.evals_per_atom() for w in batch)


@pytest.mark.parametrize("stages,stage_kb", [(3, 16), (4, 24), (3, 48)])
def test_batch_pipeline_depths(stages, stage_kb):
    """Deeper copy pipelines (3 and 4 stages in flight) give the same sums."""
    batch = _small_batch(seed=14, n=5)
    big = W.batch(nsamples=1, edge=(6, 6), nloops=(10, 10), radius=(8.0, 9.0), segments=(120, 128),
                  images=(1, 1), seed=15)[0]
    allw = batch + [big]
    us, _ = B.batch_gpu(allw, C.DISCO_FP64, stage_kb=stage_kb, stages=stages)
    for w, u in zip(allw, us):
        ref = O.displace(w.x, w.y, w.z, w.loops, w.box, images=w.images, nu=w.nu)
        assert max(np.abs(u[k] - ref[k]).max() for k in range(3)) <= 1e-9, w.name


def test_batch_rejects_bad_depth():
    batch = _small_batch(seed=16, n=2)
    with pytest.raises(C.DiscoError):
        B.batch_gpu(batch, C.DISCO_FP64, stages=5)
    with pytest.raises(C.DiscoError):
        B.batch_gpu(batch, C.DISCO_FP64, stage_kb=100, stages=3)


def test_batch_near_list_and_its_overflow():
    """FP32C batches with every pair near the cut: the FP64 pass over the
    listed (sample, atom) pairs, and, beyond the list's 2^21 entries, the
    unit-schedule FP64 pass, both reproduce the FP64 batch."""
    small = _small_batch(seed=14, n=4)
    big = W.batch(nsamples=3, edge=(80, 80), nloops=(1, 1), radius=(6.0, 8.0), segments=(16, 16),
                  images=(1, 1), seed=15)                                # 3 x 1 024 000 atoms > 2^21
    for batch in (small, big):
        u64, _ = B.batch_gpu(batch, C.DISCO_FP64)
        u32, _ = B.batch_gpu(batch, C.DISCO_FP32C, near_plane=1e6, near_rim=1e6)
        for a, b in zip(u64, u32):
            assert max(np.abs(a[k] - b[k]).max() for k in range(3)) <= 1e-12
