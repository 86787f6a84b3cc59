"""Field compatibility: the reference passes ``ti.field`` objects between its
classes (forward_modeling.py:142-149, 533-537; rtm.py:904-972).  Here a
"field" may be a torch tensor, a NumPy array, or any object with
``to_numpy()`` (a real Taichi field included); results are handed back as
``DeviceField`` objects that keep the data on the GPU and offer the same
``to_numpy()`` / ``from_numpy()`` / ``shape`` surface."""
import numpy as np
import torch


class DeviceField:
    """A device-resident array with the part of the ti.field interface the
    reference uses.  ``tensor`` is the torch view in the reference's shape."""

    def __init__(self, tensor, owner=None):
        self.tensor = tensor
        self._owner = owner  # keeps the storage behind a strided view alive

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return self.tensor.dtype

    def to_numpy(self):
        return self.tensor.detach().cpu().numpy().copy()

    def to_torch(self, device=None):
        return self.tensor if device is None else self.tensor.to(device)

    def from_numpy(self, arr):
        self.tensor.copy_(torch.as_tensor(np.asarray(arr)).to(self.tensor.dtype))

    def __getitem__(self, idx):
        v = self.tensor[idx]
        return v.item() if v.dim() == 0 else v

    def __array__(self, dtype=None, copy=None):
        a = self.to_numpy()
        return a if dtype is None else a.astype(dtype)


def to_tensor(x, dtype, device):
    """Accept a torch tensor, a DeviceField, an object with to_numpy(), or
    anything NumPy can read; return a contiguous tensor on ``device``."""
    if x is None:
        return None
    if isinstance(x, DeviceField):
        x = x.tensor
    elif not isinstance(x, torch.Tensor):
        if hasattr(x, "to_numpy"):
            x = x.to_numpy()
        x = torch.as_tensor(np.asarray(x))
    return x.to(device=device, dtype=dtype).contiguous()


def to_numpy(x, dtype=None):
    if isinstance(x, DeviceField):
        a = x.to_numpy()
    elif isinstance(x, torch.Tensor):
        a = x.detach().cpu().numpy()
    elif hasattr(x, "to_numpy"):
        a = x.to_numpy()
    else:
        a = np.asarray(x)
    return a if dtype is None else a.astype(dtype, copy=False)
