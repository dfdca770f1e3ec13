"""Data-parallel layer (atomicorbitalkernels.jl_b200/parallel.py) on CPU ranks.

Two `gloo` ranks each take a contiguous shard of a 2C batch, compute the
(zeta, D) gradient of their shard (here with the FP64 oracle, standing in for
the device pullback) and all-reduce it; the sum must equal the full-batch
gradient.  No GPU is involved.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import aok_b200 as aok
import oracle
from aok_b200 import parallel

W = aok.workloads


def test_shard_bounds_cover_the_batch():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            spans = [parallel.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        parallel.shard_bounds(10, 2, 2)


def test_shard_slices_the_last_axis():
    x = torch.arange(2 * 3 * 10).reshape(2, 3, 10)
    parts = [parallel.shard(x, r, 3) for r in range(3)]
    assert torch.equal(torch.cat(parts, dim=-1), x)


def test_allreduce_without_group_is_identity():
    a, b = torch.ones(3), torch.zeros(2, 2)
    out = parallel.allreduce_sum([a, b])
    assert out[0] is a and out[1] is b


def _problem():
    b = W.config0_basis(nspecies=2)
    pr = W.ragged_pairs(97, 2, 5)
    rng = np.random.default_rng(3)
    dS = rng.standard_normal((b.nbf_total, b.nbf_total, pr.B))
    return b, pr, dS


def _oracle_pullback(b):
    def pb(dS_local, orb, XA_local, XB_local, ps, st):
        (posA, sA), (posB, sB) = XA_local, XB_local
        dz, dD = oracle.overlap_pullback_ps(dS_local, b.ls, b.zeta, b.D, sA, sB, posA, posB)
        return {"Rnl": {"zeta": torch.as_tensor(dz), "D": torch.as_tensor(dD)}, "Ylm": {}}
    return pb


def _rank(rank, world, port, out_path):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        b, pr, dS = _problem()
        lo, hi = parallel.shard_bounds(pr.B, rank, world)
        XA = (pr.posA[:, lo:hi], pr.sidxA[lo:hi])
        XB = (pr.posB[:, lo:hi], pr.sidxB[lo:hi])
        g = parallel.overlap_pullback_ps(dS[:, :, lo:hi], None, XA, XB, None, None, pullback=_oracle_pullback(b))
        if rank == 0:
            np.savez(out_path, dz=g["Rnl"]["zeta"].numpy(), dD=g["Rnl"]["D"].numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_gradient_equals_full_batch(tmp_path):
    out = str(tmp_path / "g.npz")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    b, pr, dS = _problem()
    dz, dD = oracle.overlap_pullback_ps(dS, b.ls, b.zeta, b.D, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    for a, ref in ((got["dz"], dz), (got["dD"], dD)):
        assert np.linalg.norm(a - ref) <= 1e-12 * np.linalg.norm(ref)


def _eval_problem():
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    X, sidx = W.config1_points(nX=301, seed=9)
    dP = np.random.default_rng(4).standard_normal((301, len(orb)))
    return b, orb, X, sidx, dP


def _eval_rank(rank, world, port, out_path):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        b, orb, X, sidx, dP = _eval_problem()
        lo, hi = parallel.shard_bounds(X.shape[1], rank, world)

        def pb(dP_local, basis, X_local, ps, st):  # the oracle stands in for the device pullback
            Xl, sl = X_local
            dz, dD = oracle.evaluate_pb(dP_local, Xl, sl, b.zeta, b.D, basis.Rnl.powers(), basis.radidx,
                                        basis.ylmidx, basis.L)
            return {"Rnl": {"zeta": torch.as_tensor(dz), "D": torch.as_tensor(dD)}, "Ylm": {}}

        g = parallel.evaluate_pullback_ps(dP[lo:hi], orb, (np.asfortranarray(X[:, lo:hi]), sidx[lo:hi]), None, None,
                                          pullback=pb)
        np.savez(f"{out_path}.{rank}.npz", dz=g["Rnl"]["zeta"].numpy(), dD=g["Rnl"]["D"].numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_evaluate_gradient_equals_full_batch(tmp_path):
    """Three ranks, uneven shards of 301 points: every rank ends with the full-batch
    (zeta, D) gradient of the orbital evaluation."""
    out = str(tmp_path / "e")
    mp.spawn(_eval_rank, args=(3, _free_port(), out), nprocs=3, join=True)
    b, orb, X, sidx, dP = _eval_problem()
    dz, dD = oracle.evaluate_pb(dP, X, sidx, b.zeta, b.D, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L)
    for r in range(3):
        got = np.load(f"{out}.{r}.npz")
        for a, ref in ((got["dz"], dz), (got["dD"], dD)):
            assert np.linalg.norm(a - ref) <= 1e-12 * np.linalg.norm(ref)
