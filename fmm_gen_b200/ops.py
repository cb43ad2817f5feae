"""PyTorch custom ops over the C ABI.

``torch.ops.fmm.gemm(A, B, C, levels, pack)``: C += A @ B in place on CUDA FP64 column-major
tensors (stride(0) == 1), enqueued on the current stream through ``fmm_dgemm_dev``.  ``levels``
names the composed plan with the generator's job naming, e.g. ``"222-1"`` or ``"222-1_333-1"``;
plans are created once and cached.  ``pack`` is ``"abc"``, ``"ab"`` or ``"naive"``; ``x`` is the value of the approximate algorithms'
parameter when a level uses one.

``torch.ops.fmm.plain_gemm(A, B, C)``: the classical C += A @ B.
"""
from __future__ import annotations

import re
from typing import Optional

import torch

from . import runtime

_plans = {}


def parse_levels(levels: str):
    """'222-1_333-1' -> (['222', '333'], [1, 1])"""
    algs, lv = [], []
    for part in levels.split("_"):
        m = re.fullmatch(r"(.+)-(\d+)", part)
        if not m:
            raise ValueError(f"bad level string {levels!r}")
        algs.append(m.group(1))
        lv.append(int(m.group(2)))
    return algs, lv


def plan_for(levels: str, x: Optional[float] = None) -> runtime.Plan:
    p = _plans.get((levels, x))
    if p is None:
        p = runtime.Plan.from_levels(*parse_levels(levels), x=x)
        _plans[(levels, x)] = p
    return p


@torch.library.custom_op("fmm::gemm", mutates_args=("C",))
def gemm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, levels: str, pack: str = "abc",
         x: Optional[float] = None) -> None:
    runtime.fmm_gemm(plan_for(levels, x), A, B, C, pack)


@torch.library.custom_op("fmm::plain_gemm", mutates_args=("C",))
def plain_gemm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor) -> None:
    runtime.plain_gemm(A, B, C)
