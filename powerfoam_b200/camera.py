"""Camera of the rendering path (pinhole, or generic through ray maps).

TorchCamera keeps the fields and helpers of the reference's TorchCamera
(powerfoam/camera.py:181-305): ``eye``, ``right``, ``up`` with
|up| = tan(vfov/2), |right| = |up| * width / height and the view direction
normalize(cross(up, right)).  The open3d export of the reference is not part
of the rendering path and is not provided.
"""

from dataclasses import dataclass, field

import math

import torch

from . import _lib


@dataclass
class TorchCamera:
    eye: torch.Tensor
    right: torch.Tensor
    up: torch.Tensor
    width: int
    height: int
    ray_maps: torch.Tensor = None
    fov_cos_cutoff: float = None
    _pf: tuple = field(default=None, repr=False, compare=False)

    def to_pf(self):
        """The C-ABI pf_camera struct.  Kept while eye / right / up are the
        same tensors at the same version, so that repeated calls (and CUDA
        graph capture, where a device-to-host read is not allowed) do not
        read device tensors back."""
        key = (self.width, self.height) + tuple((id(t), t._version) for t in (self.eye, self.right, self.up))
        if self._pf is None or self._pf[0] != key:
            self._pf = (key, _lib.make_camera(self.eye, self.right, self.up, self.width, self.height))
        return self._pf[1]

    def to_device(self, device):
        dev = torch.device(device)
        return TorchCamera(
            eye=self.eye.to(dev),
            right=self.right.to(dev),
            up=self.up.to(dev),
            width=self.width,
            height=self.height,
            ray_maps=self.ray_maps.to(dev) if self.ray_maps is not None else None,
            fov_cos_cutoff=self.fov_cos_cutoff,
        )

    def get_ray_dir(self, i, j):
        """Unnormalised ray directions of pixels (i, j) (camera.py:19-24)."""
        forward = torch.cross(self.up, self.right, dim=-1)
        forward = forward / torch.norm(forward, dim=-1, keepdim=True)
        x = 2.0 * j / (float(self.width) - 1.0) - 1.0
        y = 1.0 - 2.0 * i / (float(self.height) - 1.0)
        return x[:, None] * self.right[None, :] + y[:, None] * self.up[None, :] + forward[None, :]

    def build_pinhole_ray_maps(self):
        """(H, W, 6) origins and unit directions of the pinhole rays, the ray
        maps the reference builds when none are given (camera.py:198-215)."""
        d = self.ray_directions().reshape(-1, 3)
        o = self.eye[None, :].expand(d.shape[0], 3)
        return torch.cat([o, d], dim=-1).view(self.height, self.width, 6)

    def ray_directions(self):
        """(H, W, 3) unit ray directions."""
        i = torch.arange(self.height, dtype=self.eye.dtype, device=self.eye.device)
        j = torch.arange(self.width, dtype=self.eye.dtype, device=self.eye.device)
        ii, jj = torch.meshgrid(i, j, indexing="ij")
        d = self.get_ray_dir(ii.reshape(-1), jj.reshape(-1))
        d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
        return d.view(self.height, self.width, 3)

    def intrinsics_matrix(self):
        right_norm = torch.linalg.norm(self.right) + 1e-8
        up_norm = torch.linalg.norm(self.up) + 1e-8
        fx = 0.5 * (float(self.width) - 1.0) / right_norm
        fy = 0.5 * (float(self.height) - 1.0) / up_norm
        cx = 0.5 * (float(self.width) - 1.0)
        cy = 0.5 * (float(self.height) - 1.0)
        return torch.tensor([[fx, 0.0, cx], [0.0, fy, cy], [0.0, 0.0, 1.0]], dtype=self.eye.dtype,
                            device=self.eye.device)

    def w2c(self):
        r = self.right / (torch.linalg.norm(self.right) + 1e-8)
        u = self.up / (torch.linalg.norm(self.up) + 1e-8)
        f = torch.cross(u, r, dim=-1)
        f = f / torch.linalg.norm(f + 1e-8)
        u = torch.cross(f, r, dim=-1)
        u = u / torch.linalg.norm(u + 1e-8)
        R = torch.stack([r, u, f], dim=0)
        t = -R @ self.eye
        M = torch.eye(4, dtype=self.eye.dtype, device=self.eye.device)
        M[:3, :3] = R
        M[:3, 3] = t
        return M

    def c2w(self):
        r = self.right / torch.linalg.norm(self.right)
        u = self.up / torch.linalg.norm(self.up)
        f = torch.cross(u, r, dim=-1)
        f = f / torch.linalg.norm(f)
        u = torch.cross(f, r, dim=-1)
        u = u / torch.linalg.norm(u)
        M = torch.eye(4, dtype=self.eye.dtype, device=self.eye.device)
        M[:3, :3] = torch.stack([r, u, f], dim=1)
        M[:3, 3] = self.eye
        return M

    def projection_matrix(self):
        return self.intrinsics_matrix() @ self.w2c()[:3, :]


def look_at(eye, target, width, height, vfov_deg, world_up=(0.0, 1.0, 0.0), device="cpu"):
    """Camera at ``eye`` looking at ``target`` with vertical field of view
    ``vfov_deg``; world up +y.  right = normalize(f x up_w) * tan(vfov/2) * W/H,
    up = (right_hat x f) * tan(vfov/2), so that f is normalize(cross(up, right))."""
    e = torch.as_tensor(eye, dtype=torch.float64)
    f = torch.as_tensor(target, dtype=torch.float64) - e
    f = f / f.norm()
    r = torch.linalg.cross(f, torch.as_tensor(world_up, dtype=torch.float64))
    r = r / r.norm()
    u = torch.linalg.cross(r, f)
    th = math.tan(math.radians(vfov_deg) / 2)
    return TorchCamera(
        eye=e.float().to(device),
        right=(r * th * width / height).float().to(device),
        up=(u * th).float().to(device),
        width=int(width),
        height=int(height),
    )
