"""Resume and checkpoints of the host-driven refinement: a refinement stopped
by an interrupt, continued in the same handle or written to a file and
continued by a fresh handle, reports exactly what the uninterrupted
refinement reports."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("evaluated", "verdicts", "unresolved", "clipped", "fp32_decided", "per_depth", "handles_evaluated", "digest")


# (0, 1): the start family with a lambda-only split carries its parents'
# lambda-independent terms in the levels; a checkpoint does not hold them, so
# the resumed boxes recompute them
@pytest.mark.parametrize("family,policy", [(3, 2), (5, 1), (4, 0), (0, 1)])
def test_interrupt_resume_and_checkpoint(cp, tmp_path, family, policy):
    d = cp.DIMS[family]
    kw = dict(policy=policy, max_depth=8 if policy else 3, seed_sizes=[16, 8, 8, 4][:d], level_capacity=1 << 16,
              digest=True)
    p = cp.Prover(0)
    try:
        want = p.refine(family, **kw)
        assert want["launches"] > 2  # several chunks, so an interrupt lands between them
        # an interrupt requested while no refinement runs does not stop the next one
        p.interrupt()
        again = p.refine(family, **kw)
        for k in KEYS:
            assert again[k] == want[k], k
        # same handle: interrupt after the first chunk (from the progress callback), then resume
        seen = []

        def stop_after_first(evaluated, waiting):
            if not seen:
                p.interrupt()
            seen.append((evaluated, waiting))

        p.set_chunk_callback(stop_after_first)
        with pytest.raises(cp.ProverError) as e:
            p.refine(family, **kw)
        assert e.value.status == 8  # CP_ERR_INTERRUPTED
        assert len(seen) == 1 and 0 < seen[0][0] < want["evaluated"]
        p.set_chunk_callback(None)
        got = p.refine_resume()
        for k in KEYS:
            assert got[k] == want[k], k
        with pytest.raises(cp.ProverError):
            p.refine_resume()  # nothing left to resume
        # checkpoint: interrupt, save, continue in a new handle
        seen.clear()
        p.set_chunk_callback(stop_after_first)
        with pytest.raises(cp.ProverError):
            p.refine(family, **kw)
        p.set_chunk_callback(None)
        path = tmp_path / "refine.ckpt"
        p.checkpoint_save(str(path))
    finally:
        p.close()
    q = cp.Prover(0)
    try:
        o = q.checkpoint_load(str(path))
        assert o.family == family and o.policy == policy and o.max_depth == kw["max_depth"]
        got = q.refine_resume()
        for k in KEYS:
            assert got[k] == want[k], k
    finally:
        q.close()


def test_checkpoint_rejects_foreign_files(cp, tmp_path):
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(b"not a checkpoint" * 8)
    q = cp.Prover(0)
    try:
        with pytest.raises(cp.ProverError):
            q.checkpoint_load(str(bad))
        with pytest.raises(cp.ProverError):
            q.checkpoint_save(str(tmp_path / "x.ckpt"))  # nothing interrupted
    finally:
        q.close()
