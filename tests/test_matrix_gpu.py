"""Matrix-level entry points (tblis_matrix_mult, stra_tblis_matrix_mult[_naive|_ab],
stra_tblis_matrix_mult_2level[_naive|_ab]; the reference's src/stra_iface/3m)
through the C ABI, against the oracle: C = alpha*A*B + beta*C for column- and
row-major and transposed-view operands, ragged sizes, device and host memory,
within the FP64 bound 4*12^L*k*2^-53*max|A|*max|B| (plus the beta term)."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


def case(m, n, k, order_a, order_b, order_c, seed):
    A = oracle.uniform((m, k), seed, order=order_a)
    B = oracle.uniform((k, n), seed + 1, order=order_b)
    C = oracle.uniform((m, n), seed + 2, order=order_c)
    return A, B, C


@pytest.mark.parametrize("impl", [1, 2, 3])
@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("orders", ["FFF", "CCC", "FCF", "CFC"])
def test_matrix_entry_points_vs_oracle(tsb, cuda, level, impl, orders):
    import torch
    m, n, k = 157, 130, 203
    A, B, C0 = case(m, n, k, *orders, seed=7 + level)
    alpha, beta = 1.5, 0.5
    R = C0.copy(order="A")
    oracle.contract(alpha, A, "ik", B, "kj", beta, R, "ij")

    def dev(X):
        return torch.from_numpy(X).to(cuda) if X.flags.c_contiguous else \
            torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda).T
    dA, dB, dC = dev(A), dev(B), dev(C0)
    assert list(dA.stride()) == [s // 8 for s in A.strides]
    tsb.matrix_mult(level, alpha, dA, dB, beta, dC, impl=impl)
    torch.cuda.synchronize()
    bound = abs(alpha) * oracle.error_bound(level, k, 1.0, 1.0) + 4 * 2.0 ** -53 * abs(beta)
    assert np.abs(dC.cpu().numpy() - R).max() <= bound


def test_matrix_transposed_view_and_host_memory(tsb, cuda):
    """A transposed view (rs > cs) in host memory: staged through the device."""
    m, n, k = 96, 80, 300
    At = oracle.uniform((k, m), 3)          # A = At.T: strides (k... ) of a view
    A = At.T
    B = oracle.uniform((k, n), 4)
    C = np.zeros((m, n), order="F")
    tsb.matrix_mult(1, 1.0, A, B, 0.0, C)
    R = np.zeros((m, n), order="F")
    oracle.contract(1.0, np.asfortranarray(A), "ik", B, "kj", 0.0, R, "ij")
    assert np.abs(C - R).max() <= oracle.error_bound(1, k, 1.0, 1.0)


def test_matrix_matches_tensor_entry_point(tsb, cuda):
    """The matrix call is the 2-D contraction: identical result to the tensor
    call on the same data, level and variant."""
    import torch
    m, n, k = 512, 384, 640
    A, B, C0 = case(m, n, k, "F", "F", "F", 21)
    d = lambda X: torch.from_numpy(np.ascontiguousarray(X.T)).to(cuda).T
    dA, dB = d(A), d(B)
    C1, C2 = d(C0), d(C0)
    tsb.matrix_mult(2, 1.0, dA, dB, 1.0, C1)
    tsb.contract(2, 1.0, dA, "ik", dB, "kj", 1.0, C2, "ij")
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)
