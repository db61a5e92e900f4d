"""torch.autograd binding of the weighted pair counts and their adjoint.

PairCounts.apply(w_a, w_b, ctx, cat_a, cat_b, binning, precision) returns the
raw full histogram of tpcf_count (unordered pairs for an auto count, b None)
as a float64 tensor, differentiable in the per-point weights: the backward
pass runs tpcf_count_backward, which replays the pair loop with the forward's
bin membership and sums dL/dw in double on the device.  Everything built from
the histograms in torch (normalisation by the weight sums, the Landy-Szalay
xi, a loss) is differentiated by torch itself.

The weights are float32 on the device (Galaxy::weight is float); the forward
uploads them into the catalogue (tpcf_catalog_set_weights) before counting.
"""
from __future__ import annotations

import numpy as np
import torch

from . import FP32_GUARD, count, count_backward


class PairCounts(torch.autograd.Function):
    @staticmethod
    def forward(fctx, w_a, w_b, ctx, cat_a, cat_b, binning, precision=FP32_GUARD):
        cat_a.set_weights(w_a.detach().to("cpu", torch.float32).numpy())
        if cat_b is not None:
            cat_b.set_weights(w_b.detach().to("cpu", torch.float32).numpy())
        full, _, _ = count(ctx, cat_a, cat_b, binning, precision, with_regions=False)
        fctx.objs = (ctx, cat_a, cat_b, binning, precision)
        fctx.auto = cat_b is None
        return torch.from_numpy(full).to(w_a.device)

    @staticmethod
    def backward(fctx, grad_full):
        ctx, cat_a, cat_b, binning, precision = fctx.objs
        g = grad_full.detach().to("cpu", torch.float64).numpy()
        ga, gb, _ = count_backward(ctx, cat_a, cat_b, binning, g, precision)
        ga_t = torch.from_numpy(ga).to(grad_full.device)
        gb_t = None if fctx.auto else torch.from_numpy(gb).to(grad_full.device)
        return ga_t, gb_t, None, None, None, None, None


def pair_counts(w_a, w_b, ctx, cat_a, cat_b, binning, precision=FP32_GUARD):
    """Raw full histogram of the count of cat_a (with cat_b, or auto when cat_b
    is None) under weights w_a / w_b, differentiable in the weights."""
    if cat_b is None:
        w_b = torch.zeros(1, dtype=w_a.dtype, device=w_a.device)
    return PairCounts.apply(w_a, w_b, ctx, cat_a, cat_b, binning, precision)
