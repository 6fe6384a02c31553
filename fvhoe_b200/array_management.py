"""Named-array registry with a "cuda" backend (host side).

Same interface and errors as fvhoe/array_management.py:12-61 (`ArrayManager`):
add(name, ndarray) -> KeyError on a duplicate name, TypeError on a
non-ndarray; __call__(name) and get_numpy(name) -> KeyError on a missing
name; remove; to_dict. With backend="cuda" the arrays live on the current
CUDA device as float64 torch tensors (torch is used for device memory only);
__call__ returns the tensor and get_numpy copies it back to the host.
"""

from dataclasses import dataclass, field

import numpy as np

BACKENDS = ("numpy", "cuda")


@dataclass
class ArrayManager:
    arrays: dict = field(default_factory=dict)
    backend: str = "numpy"
    device: str = "cuda"

    def __post_init__(self):
        if self.backend not in BACKENDS:
            raise ValueError(f"unknown backend {self.backend!r}; choose one of {BACKENDS}")
        if self.backend == "cuda":
            _require_cuda()

    @property
    def using_cupy(self) -> bool:
        return False

    @property
    def using_cuda(self) -> bool:
        return self.backend == "cuda"

    def __repr__(self) -> str:
        return f"ArrayManager({self.arrays.keys()}, backend={self.backend!r})"

    def enable_cuda(self):
        _require_cuda()
        if self.backend != "cuda":
            import torch

            self.arrays = {k: torch.as_tensor(v, device=self.device) for k, v in self.arrays.items()}
            self.backend = "cuda"

    def add(self, name: str, array: np.ndarray):
        if name in self.arrays:
            raise KeyError(f"Array with name '{name}' already exists.")
        if not isinstance(array, np.ndarray):
            raise TypeError("array must be of type numpy")
        if self.backend == "cuda":
            import torch

            array = torch.from_numpy(np.ascontiguousarray(array)).to(self.device)
        self.arrays[name] = array

    def add_device(self, name: str, tensor):
        """Registers a float64 device tensor already on this manager's device
        (no copy; "cuda" backend only)."""
        if self.backend != "cuda":
            raise TypeError("add_device needs the cuda backend")
        if name in self.arrays:
            raise KeyError(f"Array with name '{name}' already exists.")
        import torch

        if not isinstance(tensor, torch.Tensor) or tensor.device.type != "cuda" or tensor.dtype != torch.float64:
            raise TypeError("add_device takes a float64 CUDA tensor")
        self.arrays[name] = tensor.contiguous()

    def _check_name(self, name: str):
        if name not in self.arrays:
            raise KeyError(f"Array with name '{name}' not found.")

    def remove(self, name: str):
        self._check_name(name)
        del self.arrays[name]

    def get_numpy(self, name: str) -> np.ndarray:
        self._check_name(name)
        arr = self.arrays[name]
        if self.backend == "cuda":
            return arr.detach().cpu().numpy()
        return arr.copy()

    def __call__(self, name: str):
        self._check_name(name)
        return self.arrays[name]

    def to_dict(self) -> dict:
        return dict(names=list(self.arrays.keys()), using_cupy=False, backend=self.backend)


def _require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the cuda backend needs a CUDA device; none is visible")
