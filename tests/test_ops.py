"""The C ABI registered as torch ops (no GPU needed: schemas and fake
implementations; the GPU tests run the real ops through the public API)."""
import torch
from torch._subclasses.fake_tensor import FakeTensorMode

import peel_mpm_b200.ops  # noqa: F401  (registers torch.ops.peelmpm)


def test_ops_are_registered_with_their_schemas():
    for name in ("sym_eig", "bin_sort", "substep"):
        assert hasattr(torch.ops.peelmpm, name), name
    schema = str(torch.ops.peelmpm.substep.default._schema)
    assert "!) planes" in schema and "!) workspace" in schema
    assert "Tensor? interface_mask" in schema and "-> ()" in schema


def test_fake_implementations_propagate_shapes():
    with FakeTensorMode(allow_non_fake_inputs=False) as mode:
        A = torch.empty(17, 3, 3, device="cuda")
        ev, V = torch.ops.peelmpm.sym_eig(A, 5)
        assert ev.shape == (17, 3) and V.shape == (17, 3, 3) and ev.device.type == "cuda"
        x = torch.empty(100, 3, device="cuda")
        keys, perm = torch.ops.peelmpm.bin_sort(x, 64, 64.0)
        assert keys.shape == (100,) and keys.dtype == torch.int64 and perm.dtype == torch.int64
        planes = torch.empty(64, 128, device="cuda")
        out = torch.ops.peelmpm.substep(planes, torch.empty(100, dtype=torch.bool, device="cuda"), None, None,
                                        torch.empty(1024, dtype=torch.uint8, device="cuda"),
                                        torch.empty(8, dtype=torch.uint8), torch.empty(8, dtype=torch.uint8), 100)
        assert out is None
