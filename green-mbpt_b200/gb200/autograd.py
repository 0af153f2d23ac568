"""The GW self-energy as a differentiable torch operation.

`gw_sigma(context, G, V=None)` returns Sigma(tau, k) of a complex128 CUDA tensor G [nts, ns, nk, nso, nso]
(and, optionally, of the half-stored integrals V) through the context's device entry points; its
backward is the library's vector-Jacobian product (gb200_gw_sigma_vjp_device), so a real functional
of Sigma can be differentiated with respect to G and V by `torch.autograd`.  P0 and W are not kept
between forward and backward: the backward recomputes them per q.  torch's gradient of a real loss L with respect to a complex tensor z = x + iy
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
    def forward(ctx, G, V, context):
        G = G.contiguous()
        if V is not None:
            V = V.contiguous()
            context.set_integrals_device(V.data_ptr(), 0, V.shape[0], stream=_stream())
        Sigma = torch.empty_like(G)
        context.gw_sigma_device(G.data_ptr(), Sigma.data_ptr(), stream=_stream())
        ctx.context = context
        ctx.with_V = V is not None
        ctx.save_for_backward(G, V)
        return Sigma

    @staticmethod
    def backward(ctx, Sb):
        G, V = ctx.saved_tensors
        Sb = Sb.contiguous()
        Gb = torch.empty_like(G)
        Vb = torch.empty_like(V) if ctx.with_V and ctx.needs_input_grad[1] else None
        ctx.context.gw_sigma_vjp_device(G.data_ptr(), Sb.data_ptr(), Gb.data_ptr(),
                                        Vb.data_ptr() if Vb is not None else 0, stream=_stream())
        return Gb, Vb, None


def gw_sigma(context, G: torch.Tensor, V: torch.Tensor | None = None) -> torch.Tensor:
    """Sigma(G, V) for complex128 CUDA tensors, differentiable in G and, when given, in the half-stored
    integrals V [nk(nk+1)/2, NQ, nao, nao] (which then replace the context's GW integrals).  Without V
    the context's integrals are used and only G carries a gradient."""
    if G.dtype != torch.complex128 or not G.is_cuda:
        raise TypeError("gw_sigma: G must be a complex128 CUDA tensor")
    if tuple(G.shape) != tuple(context.shape_G):
        raise ValueError(f"gw_sigma: G has shape {tuple(G.shape)}, the context expects {tuple(context.shape_G)}")
    if V is not None:
        d = context.dims
        shape = (d.nk * (d.nk + 1) // 2, d.NQ, d.nao, d.nao)
        if V.dtype != torch.complex128 or not V.is_cuda or tuple(V.shape) != shape:
            raise ValueError(f"gw_sigma: V must be a complex128 CUDA tensor of shape {shape}")
    return _GWSigma.apply(G, V, context)
