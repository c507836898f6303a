"""Differentiation (configuration 4): GettFunction's dA and dB are generated
contractions; checked against FP64 finite differences and the FP64 einsum
gradient."""
import numpy as np
import pytest

from tccg_b200.autograd import GettFunction, grad_contractions
from tccg_b200.spec import make_contraction

CFG4 = ("xyzw", "pxqw", "qzpy")  # C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0]
CFG4_SIZES = dict(x=64, w=64, y=64, z=64, p=32, q=32)


def test_grad_contractions_labels():
    con = make_contraction(*CFG4, CFG4_SIZES)
    dA, dB = grad_contractions(con)
    assert dA.C0.labels == list("pxqw") and dA.A0.labels == list("xyzw") and dA.B0.labels == list("qzpy")
    assert dB.C0.labels == list("qzpy") and dB.A0.labels == list("pxqw") and dB.B0.labels == list("xyzw")
    assert [i.label for i in dA.k_indices] == ["y", "z"]


def _einsum_fwd(con, A, B):
    import torch
    # tensors hold reversed shapes: einsum over reversed label strings
    r = lambda t: "".join(reversed(t.labels))
    return torch.einsum("%s,%s->%s" % (r(con.A0), r(con.B0), r(con.C0)), A, B) * con.alpha


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("bf16x3", 2e-5), ("bf16", 1e-2)])
def test_cfg4_gradients_vs_fp64(cuda, precision, tol):
    import torch
    con = make_contraction(*CFG4, CFG4_SIZES)
    g = torch.Generator(device="cuda").manual_seed(7)
    shapeA = tuple(i.size for i in reversed(con.A0.indices))
    shapeB = tuple(i.size for i in reversed(con.B0.indices))
    shapeC = tuple(i.size for i in reversed(con.C0.indices))
    dt = torch.bfloat16 if precision == "bf16" else torch.float32
    A = torch.randn(shapeA, generator=g, device="cuda").to(dt).requires_grad_()
    B = torch.randn(shapeB, generator=g, device="cuda").to(dt).requires_grad_()
    dC = torch.randn(shapeC, generator=g, device="cuda")
    C = GettFunction.apply(A, B, con, precision)
    (C * dC).sum().backward()
    A64 = A.detach().double().requires_grad_()
    B64 = B.detach().double().requires_grad_()
    C64 = _einsum_fwd(con, A64, B64)
    (C64 * dC.double()).sum().backward()
    nw = lambda x, r: (torch.linalg.vector_norm(x.double() - r) / torch.linalg.vector_norm(r)).item()
    assert nw(C, C64.detach()) <= tol
    assert nw(A.grad, A64.grad) <= tol
    assert nw(B.grad, B64.grad) <= tol

    # FP64 central finite differences (eps = 1e-6) of L = <dC, C(A, B)> on 64
    # random entries of A and of B
    rng = np.random.default_rng(0)
    eps = 1e-6
    for X, X64, grad in ((A, A64, A.grad), (B, B64, B.grad)):
        flat = X64.detach().clone().reshape(-1)
        idx = rng.choice(flat.numel(), 64, replace=False)
        fd = []
        for e in idx:
            vals = []
            for sgn in (1.0, -1.0):
                f = flat.clone()
                f[e] += sgn * eps
                Xp = f.reshape(X64.shape)
                Cp = _einsum_fwd(con, Xp, B64.detach()) if X is A else _einsum_fwd(con, A64.detach(), Xp)
                vals.append((Cp * dC.double()).sum().item())
            fd.append((vals[0] - vals[1]) / (2 * eps))
        fd = np.array(fd)
        got = grad.double().reshape(-1)[torch.as_tensor(idx, device="cuda")].cpu().numpy()
        err = np.linalg.norm(got - fd) / np.linalg.norm(fd)
        assert err <= max(tol, 1e-4), (precision, err)


@pytest.mark.gpu
def test_gradcheck_fp64_small(cuda):
    """torch.autograd.gradcheck (FP64 finite differences) through the FP64 path."""
    import torch
    con = make_contraction("abc", "kab", "ck", dict(a=5, b=3, c=4, k=6), alpha=1.5)
    A = torch.randn(6 * 5 * 3, dtype=torch.float64, device="cuda", requires_grad=True)
    B = torch.randn(4 * 6, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: GettFunction.apply(a, b, con, "fp64"), (A, B),
                                    eps=1e-6, atol=1e-8)


@pytest.mark.gpu
def test_c_input_gradient(cuda):
    import torch
    con = make_contraction("ab", "ak", "kb", dict(a=7, b=9, k=5), alpha=2.0, beta=0.5)
    A = torch.randn(5, 7, device="cuda", requires_grad=True)
    B = torch.randn(9, 5, device="cuda", requires_grad=True)
    Cin = torch.randn(9, 7, device="cuda", requires_grad=True)
    C = GettFunction.apply(A, B, con, "fp32", Cin)
    ref = 2.0 * torch.einsum("ka,bk->ba", A, B) + 0.5 * Cin
    assert torch.allclose(C, ref, rtol=1e-5, atol=1e-5)
    C.sum().backward()
    assert torch.allclose(Cin.grad, torch.full_like(Cin, 0.5))
