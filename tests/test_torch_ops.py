"""torch.ops.m3d loads and registers every operator (no GPU needed)."""
import pytest


def test_torch_ops_registered(m3d_lib):
    torch = pytest.importorskip("torch")
    from dispatch_b200 import torch_ops
    ops = torch_ops.load()
    for name in torch_ops.OPS:
        op = getattr(ops, name)
        assert op.default._schema.name == f"m3d::{name}"
    # the in-place operators declare what they write
    s = str(ops.formal_solve.default._schema)
    assert "Tensor(a!) work" in s and "Tensor(b!)? psi" in s
