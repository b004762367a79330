"""Per-resolution tuning of the frame's free parameters.

The tile shape is fixed at the reference's 16 x 16 pixels (the tile lists,
ranges and the compositor's block are defined on it), so what is tuned is how
the tile entries are sorted: the digit width of the radix passes (balanced
digits, or 4..8 bits) and the method (radix passes or the one-pass tile
transpose, where the frame has at most 16,384 tiles). Every choice produces
the same lists bit for bit; only the time differs. For each distinct viewport
of a set of views, one representative view is rendered with every candidate
and the candidate with the smallest median Stage 3 device time is kept.
"""
from __future__ import annotations

import statistics

from . import _abi

DIGIT_WIDTHS = (0, 4, 5, 6, 7, 8)


def candidates(width: int, height: int):
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    out = [(rb, _abi.SORT_RADIX) for rb in DIGIT_WIDTHS]
    if tiles <= 16384:
        out.append((0, _abi.SORT_TRANSPOSE))
    return out


def tune_views(state, scene, cages, cameras, compositors, repeats: int = 3) -> dict:
    """{(width, height): (radix_bits, entry_sort, stage3_ms)} for the
    viewports of the views; uses the first view of each viewport."""
    first = {}
    for cam, comp in zip(cameras, compositors):
        first.setdefault((comp.screen_width, comp.screen_height), (cam, comp))
    best = {}
    for key, (cam, comp) in first.items():
        results = []
        for rb, es in candidates(*key):
            # one frame to size the buffers, then the timed ones
            state.execute_frame_gpu(scene, cages, cam, comp, force_stage3=True,
                                    radix_bits=rb, entry_sort=es)
            ms = [state.execute_frame_gpu(scene, cages, cam, comp, force_stage3=True,
                                          profile_stages=True, radix_bits=rb,
                                          entry_sort=es).stage3_bin_sort_ms
                  for _ in range(repeats)]
            results.append((statistics.median(ms), rb, es))
        ms, rb, es = min(results)
        best[key] = (rb, es, ms)
    return best


def per_view(best: dict, compositors):
    """(radix_bits list, entry_sort list) for execute_views."""
    rbs, ess = [], []
    for comp in compositors:
        rb, es, _ = best[(comp.screen_width, comp.screen_height)]
        rbs.append(rb)
        ess.append(es)
    return rbs, ess
