"""The tcgen05 BF16 tensor-core GEMM (og_tc_gemm) against a float64 matmul
of the same BF16-rounded operands.  FP32 accumulation in TMEM: error below
1e-5 of sum |a||b| per output element."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(x):
    import torch
    return x.to(torch.bfloat16).to(torch.float64)


def gemm(origami, a, a_sm, a_sk, b, b_sn, b_sk, c, c_sm, c_sn, m, n, k, bias=None, act=None, splits=1):
    lib = origami.lib()
    st = lib.og_tc_gemm(a.data_ptr(), a_sm, a_sk, b.data_ptr(), b_sn, b_sk, c.data_ptr(), c_sm, c_sn, m, n, k,
                        bias.data_ptr() if bias is not None else None,
                        act.data_ptr() if act is not None else None, splits, None)
    assert st == 0, lib.og_last_error()


def check(got, ref, a_abs, b_abs):
    bound = 1e-5 * (a_abs @ b_abs.T) + 1e-30
    err = (got.double() - ref).abs()
    assert bool((err <= bound + 1e-6 * ref.abs()).all()), float((err / bound).max())


@pytest.mark.parametrize("m,n,k", [(300, 100, 200), (128, 128, 64), (129, 7, 50), (1000, 128, 128)])
def test_row_major(origami, m, n, k):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n)
    a = torch.randn(m, k, device="cuda", generator=g)
    b = torch.randn(n, k, device="cuda", generator=g)
    c = torch.full((m, n), float("nan"), device="cuda")
    gemm(origami, a, k, 1, b, k, 1, c, n, 1, m, n, k)
    torch.cuda.synchronize()
    ref = bf16(a) @ bf16(b).T
    check(c, ref, bf16(a).abs(), bf16(b).abs())


def test_transposed_operands_bias_and_silu(origami):
    import torch
    m, n, k = 200, 130, 96
    g = torch.Generator(device="cuda").manual_seed(5)
    at = torch.randn(k, m, device="cuda", generator=g)      # A stored transposed
    bt = torch.randn(k, n, device="cuda", generator=g)      # B stored transposed
    bias = torch.randn(n, device="cuda", generator=g)
    ct = torch.full((n, m), float("nan"), device="cuda")    # C written transposed
    act = torch.full((n, m), float("nan"), device="cuda")
    gemm(origami, at, 1, m, bt, 1, n, ct, 1, m, m, n, k, bias=bias, act=act)
    torch.cuda.synchronize()
    a, b = bf16(at.T), bf16(bt.T)
    ref = a @ b.T + bias.double()
    check(ct.T, ref, a.abs(), b.abs())
    want = ct.T.double() * torch.sigmoid(ct.T.double())
    assert float((act.T.double() - want).abs().max()) < 1e-5 * float(want.abs().max() + 1)


def test_split_k_matches_unsplit(origami):
    import torch
    m, n, k = 128, 64, 4096
    g = torch.Generator(device="cuda").manual_seed(9)
    a = torch.randn(m, k, device="cuda", generator=g)
    b = torch.randn(n, k, device="cuda", generator=g)
    c1 = torch.zeros(m, n, device="cuda")
    c8 = torch.zeros(m, n, device="cuda")
    gemm(origami, a, k, 1, b, k, 1, c1, n, 1, m, n, k, splits=1)
    gemm(origami, a, k, 1, b, k, 1, c8, n, 1, m, n, k, splits=8)
    torch.cuda.synchronize()
    ref = bf16(a) @ bf16(b).T
    check(c1, ref, bf16(a).abs(), bf16(b).abs())
    check(c8, ref, bf16(a).abs(), bf16(b).abs())


def test_rejects_bad_sizes(origami):
    import torch
    lib = origami.lib()
    x = torch.zeros(4, device="cuda")
    assert lib.og_tc_gemm(x.data_ptr(), 1, 1, x.data_ptr(), 1, 1, x.data_ptr(), 1, 1, 0, 1, 1, None, None, 1,
                          None) == 1
