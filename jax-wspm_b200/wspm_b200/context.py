"""Helpers shared by the reference-API shims: array conversion and mesh cache.

The reference's functions take the mesh arrays on every call
(``assemble_global_matrices_sparse_re(triangles, nnt, points, ...)``).  The
device mesh and its SELL-32 pattern are built once per (points, elements)
pair and cached, keyed by the arrays' identity and buffers, so repeated calls
from a solver's Picard loop reuse them.
"""
import numpy as np
import torch

_MESHES = {}
_MAX_MESHES = 8


def device():
    if not torch.cuda.is_available():
        raise RuntimeError("wspm_b200 needs a CUDA device; there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def as_cuda_f64(a):
    if isinstance(a, torch.Tensor):
        t = a.to(device=device(), dtype=torch.float64)
    else:
        t = torch.as_tensor(np.asarray(a, dtype=np.float64), device=device())
    return t.contiguous().reshape(-1)


def as_host(a, dtype=None):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=dtype)


def _key(a):
    if isinstance(a, torch.Tensor):
        return ("t", a.data_ptr(), tuple(a.shape), str(a.dtype))
    a = np.asarray(a)
    return ("n", a.__array_interface__["data"][0], a.shape, a.dtype.str)


def mesh_for(points, elements):
    """Cached DeviceMesh for this (points, elements) pair."""
    from .device import DeviceMesh
    k = (_key(points), _key(elements))
    dm = _MESHES.get(k)
    if dm is not None:
        ref_p, ref_e = dm._source
        if np.array_equal(ref_e, as_host(elements)) and np.array_equal(ref_p, as_host(points)):
            return dm
    p, e = as_host(points, np.float64), as_host(elements, np.int64)
    dm = DeviceMesh(p, e, device=device())
    dm._source = (p.copy(), e.copy())
    if len(_MESHES) >= _MAX_MESHES:
        _MESHES.pop(next(iter(_MESHES)))
    _MESHES[k] = dm
    return dm
