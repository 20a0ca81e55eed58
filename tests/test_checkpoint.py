"""Checkpoint and exact resume: an engine restored from a checkpoint continues its
chains bit for bit as the saved engine does (positions, identities, list order,
accept counts, tracked energies), with and without delayed acceptance.  Bit for
bit needs launch quorum 1: with a smaller quorum the rebuild points of a batched
engine depend on which replica fills its pending buffer first, so the tracked
energies of two runs differ by FP32 rounding of the reciprocal dE."""
import numpy as np
import pytest

from ph_brush_b200 import Engine, Surrogate, _abi, configs


def _replicas():
    S, P = [], []
    for k in range(3):
        s, p = configs.small_system(seed=80 + k, p_swap=0.2, salt_conc=0.05)
        S.append(s)
        P.append(p)
    return S, P


def _continue(e, trials):
    st = e.run(trials)
    return e.state(-1), [(d["attempted"], d["accepted"], d["energy"], d["n_cations"], d["n_anions"]) for d in st]


@pytest.mark.gpu
@pytest.mark.parametrize("with_surrogate", [False, True])
def test_resume_from_checkpoint_is_bit_exact(tmp_path, with_surrogate):
    S, P = _replicas()
    path = tmp_path / "engine.ckpt"
    sur = Surrogate(seed=5) if with_surrogate else None
    with Engine(S, P) as a:
        a.set_tuning(16, 256)
        a.set_quorum(1.0)
        if sur is not None:
            a.attach_surrogate(sur, threshold=0.0)
        a.run(3000)
        a.checkpoint_save(path)
        sa, ra = _continue(a, 4000)
    with Engine(S, P) as b:  # default tuning and quorum: the checkpoint restores the saved ones
        if sur is not None:
            b.attach_surrogate(sur, threshold=0.0)
        b.checkpoint_load(path)
        assert b.tuning()["pending_max"] == 16
        sb, rb = _continue(b, 4000)
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    assert ra == rb
    if sur is not None:
        sur.close()


@pytest.mark.gpu
def test_charge_mesh_kept_by_the_mc_kernel_is_a_fresh_spread_bit_for_bit(tmp_path):
    """The charge mesh is the last section of a checkpoint: after thousands of accepted
    displacements, titrations and swaps, the mesh the MC kernel kept current equals,
    byte for byte, the mesh spread from scratch for the same configuration."""
    S, P = _replicas()
    with Engine(S, P) as a, Engine(S, P) as b:
        st = a.run(20000)
        assert all(sum(d["accepted"]) > 1000 for d in st)
        a.checkpoint_save(tmp_path / "a.ckpt")
        b.set_state(a.state(-1), -1)  # full recompute: the mesh spread from the positions
        b.checkpoint_save(tmp_path / "b.ckpt")
        nq = sum(p.mesh[0] * p.mesh[1] * _band_planes(s, p) for s, p in zip(S, P))
    qa = np.fromfile(tmp_path / "a.ckpt", dtype=np.int64)[-nq:]
    qb = np.fromfile(tmp_path / "b.ckpt", dtype=np.int64)[-nq:]
    assert np.any(qa != 0)
    assert np.array_equal(qa, qb), int(np.count_nonzero(qa != qb))


def _band_planes(s, p):
    """Planes of the wall band (the engine's rule: one plane of margin either side)."""
    nz = p.mesh[2]
    g = nz / float(np.float32(s.box[2]))
    lo = int(np.floor(p.wall_lo * g)) - 1 + p.order // 2 - p.order + 1
    hi = int(np.floor(p.wall_hi * g)) + 1 + p.order // 2
    return min(nz, hi - lo + 1)


@pytest.mark.gpu
def test_checkpoint_of_other_replicas_is_refused(tmp_path):
    S, P = _replicas()
    path = tmp_path / "engine.ckpt"
    with Engine(S, P) as a:
        a.checkpoint_save(path)
    with Engine(S[:2], P[:2]) as b:
        with pytest.raises(RuntimeError):
            b.checkpoint_load(path)


def test_checkpoint_arguments_are_checked_without_a_gpu(tmp_path):
    lib = _abi.lib()
    assert lib.phmc_checkpoint_save(None, str(tmp_path / "x").encode()) != 0
    assert lib.phmc_checkpoint_load(None, str(tmp_path / "x").encode()) != 0
