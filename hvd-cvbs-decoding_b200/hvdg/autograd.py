"""torch.autograd binding of the decode and its adjoint.

`decode(ctx, samples, geometry, lambda_c, eps, eps_c, k, cfg)` decodes a batch
of fields of one geometry on the GPU (hvdg_decode_fields) and returns the luma
(n, h, w) and chroma (n, h, w, 2) as tensors; its backward runs the library's
adjoint (hvdg_decode_fields_adjoint: the forward recomputed with the IRLS
iterates checkpointed, one implicit-function adjoint CG solve per IRLS outer
on the same SPD operator), giving gradients with respect to the input
samples and the four regulariser scalars (lambda_c, charbonnier_eps,
chroma_eps, structure_coupling). The lock-in carrier phase and the
chroma-anisotropy split are held at their forward values.

torch is plumbing here: the arithmetic of both directions runs in the CUDA
library; tensors cross the boundary as host arrays.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _cabi, api

_SCALARS = ("lambda_c", "charbonnier_eps", "chroma_eps", "structure_coupling")


def _fields(samples: np.ndarray, geometry, parity, sample_type, blanking, white):
    out = []
    for i in range(samples.shape[0]):
        s = samples[i]
        if sample_type == _cabi.SAMPLES_U16:
            s = s.astype(np.uint16)
        elif sample_type == _cabi.SAMPLES_S16:
            s = s.astype(np.int16)
        else:
            s = s.astype(np.float32)
        out.append(api.Field(np.ascontiguousarray(s), geometry, parity=int(parity[i]),
                             blanking_level=blanking, white_level=white))
    return out


class _Decode(torch.autograd.Function):
    @staticmethod
    def forward(fctx, samples, lambda_c, eps, eps_c, k, hctx, geometry, cfg, parity,
                sample_type, blanking, white, adj_iters):
        vals = dict(zip(_SCALARS, (float(lambda_c), float(eps), float(eps_c), float(k))))
        c = _cabi.config_copy(cfg, **vals)
        arr = samples.detach().cpu().numpy()
        fields = _fields(arr, geometry, parity, sample_type, blanking, white)
        dec = hctx.decode_fields(fields, c)
        y = torch.from_numpy(np.stack([d.luma for d in dec])).to(samples.device)
        chi = torch.from_numpy(np.stack([d.chroma.view(np.float32).reshape(d.chroma.shape + (2,))
                                         for d in dec])).to(samples.device)
        fctx.hctx, fctx.fields, fctx.cfg, fctx.adj_iters = hctx, fields, c, adj_iters
        fctx.dtype, fctx.device = samples.dtype, samples.device
        return y, chi

    @staticmethod
    def backward(fctx, gy, gchi):
        n = len(fctx.fields)
        gy = (gy if gy is not None else torch.zeros(0)).detach().cpu().numpy()
        gc = (gchi if gchi is not None else torch.zeros(0)).detach().cpu().numpy()
        ybar, cbar = [], []
        for i, f in enumerate(fctx.fields):
            shape = (f.geometry.active_lines, f.geometry.active_width)
            ybar.append(gy[i] if gy.size else np.zeros(shape, np.float32))
            cbar.append(gc[i].astype(np.float32).view(np.complex64)[..., 0] if gc.size
                        else np.zeros(shape, np.complex64))
        sbar, sc, _ = fctx.hctx.decode_fields_adjoint(fctx.fields, fctx.cfg, ybar, cbar,
                                                      fctx.adj_iters)
        g_samples = torch.from_numpy(np.stack(sbar)).to(device=fctx.device, dtype=fctx.dtype)
        g = [torch.tensor(sc[name], dtype=torch.float64) for name in _SCALARS]
        return (g_samples, g[0], g[1], g[2], g[3], None, None, None, None, None, None, None,
                None)


def decode(hctx: api.Context, samples: torch.Tensor, geometry, lambda_c, eps, eps_c, k,
           cfg=None, parity=None, sample_type: int = _cabi.SAMPLES_F32_IRE,
           blanking: float = 16384.0, white: float = 51200.0, adjoint_cg_iterations: int = 0):
    """Differentiable 2-D decode of `samples` (n, field_height, field_width):
    returns (luma (n, h, w), chroma (n, h, w, 2)). `lambda_c`, `eps`, `eps_c`,
    `k` are scalar tensors (or floats) that may require grad. For integer
    sample types the values are codes (float tensor holding integers) and the
    sample gradient is per code. cfg.temporal_strength must be negative."""
    cfg = cfg if cfg is not None else api.default_config(temporal_strength=-1.0)
    if parity is None:
        parity = [i % 2 for i in range(samples.shape[0])]
    as_t = lambda v: v if torch.is_tensor(v) else torch.tensor(float(v), dtype=torch.float64)
    return _Decode.apply(samples, as_t(lambda_c), as_t(eps), as_t(eps_c), as_t(k), hctx,
                         geometry, cfg, list(parity), sample_type, blanking, white,
                         adjoint_cg_iterations)
