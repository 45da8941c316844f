"""Host-side pieces of the renderer (no GPU): the camera structure passed to
the C ABI follows changes to the camera's R and T, and the world map's
layout."""
import numpy as np
import torch

from peel_mpm_b200.render import Camera, world_map


def test_camera_struct_follows_in_place_and_replaced_R_T():
    c = Camera(R=np.eye(3), T=np.zeros(3), fx=100.0, fy=90.0, width=64, height=48, device="cpu")
    s = c._struct()
    assert list(s.R) == [1, 0, 0, 0, 1, 0, 0, 0, 1] and list(s.T) == [0, 0, 0]
    assert (s.fx, s.fy, s.width, s.height) == (100.0, 90.0, 64, 48)
    c.T.add_(0.5)                                  # in place
    assert list(c._struct().T) == [0.5, 0.5, 0.5]
    c.R = torch.diag(torch.tensor([2.0, 3.0, 4.0]))   # replaced
    assert list(c._struct().R) == [2, 0, 0, 0, 3, 0, 0, 0, 4]
    c.R.data = torch.diag(torch.tensor([5.0, 6.0, 7.0]))   # new storage behind the same tensor
    assert list(c._struct().R) == [5, 0, 0, 0, 6, 0, 0, 0, 7]
    del c.R                                                # a replacement that may reuse a freed id
    c.R = torch.eye(3) * 9.0
    assert list(c._struct().R) == [9, 0, 0, 0, 9, 0, 0, 0, 9]


def test_world_map_layout():
    A = np.array([[2.0, 0, 0], [0, 3.0, 0], [0, 0, 4.0]])
    t = np.array([1.0, -1.0, 0.5])
    m = world_map(A, t, "cpu")
    assert m.shape == (3, 4) and m.dtype == torch.float32 and m.is_contiguous()
    assert torch.equal(m[:, :3], torch.tensor(A, dtype=torch.float32))
    assert torch.equal(m[:, 3], torch.tensor(t, dtype=torch.float32))
    assert torch.equal(world_map(device="cpu"), torch.cat([torch.eye(3), torch.zeros(3, 1)], 1))
