"""The GW self-energy as a differentiable torch operation.

`gw_sigma(context, G)` returns Sigma(tau, k) of a complex128 CUDA tensor G [nts, ns, nk, nso, nso]
through the context's device entry point; its backward is the library's vector-Jacobian product
(gb200_gw_sigma_vjp_device), so a real functional of Sigma can be differentiated with respect to G
by `torch.autograd`.  torch's gradient of a real loss L with respect to a complex tensor z = x + iy
is dL/dx + i dL/dy; the library's product Gb of a cotangent Sb satisfies
dL = Re sum conj(Gb) dG for L = Re sum conj(Sb) Sigma, which is the same convention, so the cotangent
passes through unchanged.  The forward runs at the context's precision, the backward in FP64.
"""
from __future__ import annotations

import torch


_CUDA_STREAM_LEGACY = 0x1  # the runtime's handle of the legacy default stream


def _stream() -> int:
    """torch's current stream as a handle for the library: a null handle would select the
    context's own (non-blocking) stream, so torch's default stream is passed by its legacy handle."""
    h = torch.cuda.current_stream().cuda_stream
    return h if h else _CUDA_STREAM_LEGACY


class _GWSigma(torch.autograd.Function):
    @staticmethod
    def forward(ctx, G, context):
        G = G.contiguous()
        Sigma = torch.empty_like(G)
        context.gw_sigma_device(G.data_ptr(), Sigma.data_ptr(), stream=_stream())
        ctx.context = context
        ctx.save_for_backward(G)
        return Sigma

    @staticmethod
    def backward(ctx, Sb):
        (G,) = ctx.saved_tensors
        Sb = Sb.contiguous()
        Gb = torch.empty_like(G)
        ctx.context.gw_sigma_vjp_device(G.data_ptr(), Sb.data_ptr(), Gb.data_ptr(), stream=_stream())
        return Gb, None


def gw_sigma(context, G: torch.Tensor) -> torch.Tensor:
    """Sigma(G) for a complex128 CUDA tensor of the context's G shape, differentiable in G."""
    if G.dtype != torch.complex128 or not G.is_cuda:
        raise TypeError("gw_sigma: G must be a complex128 CUDA tensor")
    if tuple(G.shape) != tuple(context.shape_G):
        raise ValueError(f"gw_sigma: G has shape {tuple(G.shape)}, the context expects {tuple(context.shape_G)}")
    return _GWSigma.apply(G, context)
