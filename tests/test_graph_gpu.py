"""Graph mode of the fixed-basis 2C forward (aok_plan_set_graph): the launch
chain replayed from one CUDA graph must give bitwise the results of direct
launches, also after its arguments change (re-capture with a graph update),
after the basis is replaced, and with timing enabled (direct launches)."""
import ctypes

import numpy as np
import pytest
import torch

import aok_b200 as aok
from aok_b200 import _dev, _lib

pytestmark = pytest.mark.gpu
W = aok.workloads


def _forward(L, plan, out, c, B, ls=1.0):
    _lib.check(L.aok_overlap2c(plan.h, _dev.ptr(out), None, None, _dev.ptr(c["pA"]), _dev.ptr(c["pB"]),
                               ctypes.c_void_p(c["sA"].data_ptr()), ctypes.c_void_p(c["sB"].data_ptr()), B, ls,
                               _dev.stream()))


@pytest.mark.parametrize("FT", [torch.float32, torch.float64])
def test_graph_replay_matches_direct(FT):
    L = _lib.load()
    b = W.config2_basis()
    pr = W.ragged_pairs(3000, b.NZ, 77)
    N, B = b.nbf_total, pr.B
    plan = _dev.Plan(b.ls, b.K, b.NZ, _dev.prec_of(FT), B)
    zeta = _dev.to_colmajor(b.zeta, FT)
    D = _dev.to_colmajor(b.D, FT)
    coef = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
    _lib.check(L.aok_plan_set_basis(plan.h, _dev.ptr(zeta), _dev.ptr(coef), _dev.stream()))
    c = dict(pA=_dev.to_colmajor(pr.posA, FT), pB=_dev.to_colmajor(pr.posB, FT),
             sA=torch.as_tensor(pr.sidxA).cuda(), sB=torch.as_tensor(pr.sidxB).cuda())

    ref = _dev.colmajor_empty((N, N, B), FT)
    _forward(L, plan, ref, c, B)                      # direct launches
    ref_half = _dev.colmajor_empty((N, N, B // 2), FT)
    _forward(L, plan, ref_half, c, B // 2)
    ref_ls = _dev.colmajor_empty((N, N, B), FT)
    _forward(L, plan, ref_ls, c, B, 1.25)

    _lib.check(L.aok_plan_set_graph(plan.h, 1))
    o1 = _dev.colmajor_empty((N, N, B), FT)
    o2 = _dev.colmajor_empty((N, N, B), FT)
    for _ in range(3):                                 # capture, then replays
        o1.fill_(float("nan"))
        _forward(L, plan, o1, c, B)
        torch.cuda.synchronize()
        assert torch.equal(o1, ref)
    _forward(L, plan, o2, c, B)                        # new output pointer: re-capture
    oh = _dev.colmajor_empty((N, N, B // 2), FT)
    _forward(L, plan, oh, c, B // 2)                   # new batch size
    ol = _dev.colmajor_empty((N, N, B), FT)
    _forward(L, plan, ol, c, B, 1.25)                  # new lengthscale
    o1.fill_(float("nan"))
    _forward(L, plan, o1, c, B)                        # back to the first arguments
    torch.cuda.synchronize()
    assert torch.equal(o2, ref) and torch.equal(oh, ref_half) and torch.equal(ol, ref_ls)
    assert torch.equal(o1, ref)

    # new basis parameters: the graph reads the plan's records, so it follows them
    z2 = zeta * 1.1
    c2 = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(c2), _dev.ptr(z2), _dev.ptr(D), _dev.stream()))
    _lib.check(L.aok_plan_set_basis(plan.h, _dev.ptr(z2), _dev.ptr(c2), _dev.stream()))
    _forward(L, plan, o1, c, B)
    _lib.check(L.aok_plan_set_graph(plan.h, 0))
    _forward(L, plan, o2, c, B)
    torch.cuda.synchronize()
    assert torch.equal(o1, o2) and not torch.equal(o1, ref)

    # timing enabled: direct launches, same results
    _lib.check(L.aok_plan_set_graph(plan.h, 1))
    _lib.check(L.aok_plan_timing_enable(plan.h, 4))
    o1.fill_(float("nan"))
    _forward(L, plan, o1, c, B)
    tot, n = ctypes.c_double(), ctypes.c_int64()
    _lib.check(L.aok_plan_timing_read(plan.h, ctypes.byref(tot), ctypes.byref(n)))
    assert n.value == 1 and torch.equal(o1, o2)
    _lib.check(L.aok_plan_check(plan.h, _dev.stream()))


@pytest.mark.parametrize("FT", [torch.float32, torch.float64])
def test_autotune_keeps_results_and_caches(FT):
    """aok_plan_autotune: every candidate shape computes the same blocks (the schedule
    only reorders work), the chosen shape is reported, and a second plan with the same
    key takes it from the process-wide cache."""
    L = _lib.load()
    b = W.config2_basis()
    pr = W.ragged_pairs(2500, b.NZ, 91)
    N, B = b.nbf_total, pr.B
    zeta = _dev.to_colmajor(b.zeta, FT)
    D = _dev.to_colmajor(b.D, FT)
    c = dict(pA=_dev.to_colmajor(pr.posA, FT), pB=_dev.to_colmajor(pr.posB, FT),
             sA=torch.as_tensor(pr.sidxA).cuda(), sB=torch.as_tensor(pr.sidxB).cuda())
    outs, choices = [], []
    for _ in range(2):
        plan = _dev.Plan(b.ls, b.K, b.NZ, _dev.prec_of(FT), B)
        coef = _dev.colmajor_empty(b.zeta.shape, FT)
        _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
        ref = _dev.colmajor_empty((N, N, B), FT)
        _lib.check(L.aok_overlap2c(plan.h, _dev.ptr(ref), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(c["pA"]),
                                   _dev.ptr(c["pB"]), ctypes.c_void_p(c["sA"].data_ptr()),
                                   ctypes.c_void_p(c["sB"].data_ptr()), B, 1.0, _dev.stream()))
        out = _dev.colmajor_empty((N, N, B), FT)
        ch = (ctypes.c_int64 * 3)()
        _lib.check(L.aok_plan_autotune(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(c["pA"]),
                                       _dev.ptr(c["pB"]), ctypes.c_void_p(c["sA"].data_ptr()),
                                       ctypes.c_void_p(c["sB"].data_ptr()), B, 1.0, _dev.stream(), ch))
        assert torch.equal(out, ref)
        out2 = _dev.colmajor_empty((N, N, B), FT)
        _forward(L, plan, out2, c, B)  # the basis stays fixed in the tuned plan
        torch.cuda.synchronize()
        assert torch.equal(out2, ref)
        outs.append(ref)
        choices.append(tuple(ch))
    ctas, stage, cached = choices[0]
    assert ctas in ((1, 2) if FT == torch.float64 else (2, 3)) and stage > 0
    assert choices[1][:2] == choices[0][:2] and choices[1][2] == 1


@pytest.mark.parametrize("FT,tol", [(torch.float32, 2e-6), (torch.float64, 1e-12)])
def test_autotune_cheap_items_matches_oracle(FT, tol):
    """A basis of one primitive per shell (s and p shells only: cheap items, where the
    tuner may deal a segment's items to the warps in a fixed order instead of claiming
    them): the tuned forward equals the untuned one bitwise and the oracle to the
    precision's bar."""
    import oracle
    from helpers import f32_round, rel_fro
    L = _lib.load()
    b = W.outputbound_sp_basis()
    pr = W.ragged_pairs(3000, b.NZ, 93)
    N, B = b.nbf_total, pr.B
    zeta = _dev.to_colmajor(b.zeta, FT)
    D = _dev.to_colmajor(b.D, FT)
    c = dict(pA=_dev.to_colmajor(pr.posA, FT), pB=_dev.to_colmajor(pr.posB, FT),
             sA=torch.as_tensor(pr.sidxA).cuda(), sB=torch.as_tensor(pr.sidxB).cuda())
    plan = _dev.Plan(b.ls, b.K, b.NZ, _dev.prec_of(FT), B)
    coef = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
    ref = _dev.colmajor_empty((N, N, B), FT)
    _lib.check(L.aok_overlap2c(plan.h, _dev.ptr(ref), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(c["pA"]),
                               _dev.ptr(c["pB"]), ctypes.c_void_p(c["sA"].data_ptr()),
                               ctypes.c_void_p(c["sB"].data_ptr()), B, 1.0, _dev.stream()))
    out = _dev.colmajor_empty((N, N, B), FT)
    _lib.check(L.aok_plan_autotune(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(c["pA"]),
                                   _dev.ptr(c["pB"]), ctypes.c_void_p(c["sA"].data_ptr()),
                                   ctypes.c_void_p(c["sB"].data_ptr()), B, 1.0, _dev.stream(), None))
    assert torch.equal(out, ref)
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    coef_h = coef.double().cpu().numpy()
    o = oracle.overlap2c_orb(b.ls, coef_h, rnd(b.zeta), pr.sidxA, pr.sidxB, rnd(pr.posA), rnd(pr.posB), nthreads=8)
    assert rel_fro(out.double().cpu().numpy(), o) < tol
