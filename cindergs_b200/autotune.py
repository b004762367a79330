"""Per-resolution tuning of the frame's free parameters, and of its kernels'
launch shapes.

Three parameters are tuned per viewport: the screen tile shape of Stages 3
and 4 (the reference's 16 x 16 pixels, 8 x 8 or 32 x 16: larger tiles give
fewer tile entries to bin and sort but more candidate splats per pixel in
the compositor), and how the tile entries are sorted -- the digit width of
the radix passes (balanced digits, or 4..8 bits) and the method (radix
passes or the one-pass tile transpose, where the frame has at most 16,384
tiles). The sort choices produce the same lists bit for bit; the tile shape
changes a pixel only where the tile test's rounding admits a splat whose
alpha is below the 1/255 cut there anyway. For each distinct viewport of a
set of views, one representative view is rendered with every candidate and
the candidate with the smallest median Stage 3 + Stage 4 device time is
kept.

Launch shapes (`tune_launch_shape`): the Stage 2 block size (128, 256 or 512
threads), the binning kernel's resident blocks per SM (1 or 2) and the
tile-range kernel's grid are tuned one after another (coordinate descent,
each over the others' current best) on one view, by the median Stage 2 + 3 +
4 device time; every shape gives the same frame bit for bit.
"""
from __future__ import annotations

import statistics

from . import _abi

DIGIT_WIDTHS = (0, 4, 5, 6, 7, 8)
TILE_SHAPES = (_abi.TILE_16X16, _abi.TILE_8X8, _abi.TILE_32X16)


def candidates(width: int, height: int, tile_shapes=TILE_SHAPES):
    """(tile_shape, radix_bits, entry_sort) triples worth timing."""
    out = []
    for ts in tile_shapes:
        tw, th = _abi.TILE_SHAPES[ts]
        tiles = ((width + tw - 1) // tw) * ((height + th - 1) // th)
        out += [(ts, rb, _abi.SORT_RADIX) for rb in DIGIT_WIDTHS]
        if tiles <= 16384:
            out.append((ts, 0, _abi.SORT_TRANSPOSE))
    return out


def tune_views(state, scene, cages, cameras, compositors, repeats: int = 3,
               tile_shapes=TILE_SHAPES) -> dict:
    """{(width, height): (tile_shape, radix_bits, entry_sort, stage34_ms)} for
    the viewports of the views; uses the first view of each viewport."""
    first = {}
    for cam, comp in zip(cameras, compositors):
        first.setdefault((comp.screen_width, comp.screen_height), (cam, comp))
    best = {}
    for key, (cam, comp) in first.items():
        results = []
        for ts, rb, es in candidates(*key, tile_shapes=tile_shapes):
            # one frame to size the buffers, then the timed ones
            state.execute_frame_gpu(scene, cages, cam, comp, force_stage3=True,
                                    radix_bits=rb, entry_sort=es, tile_shape=ts)
            ms = []
            for _ in range(repeats):
                t = state.execute_frame_gpu(scene, cages, cam, comp, force_stage3=True,
                                            profile_stages=True, radix_bits=rb, entry_sort=es,
                                            tile_shape=ts)
                ms.append(t.stage3_bin_sort_ms + t.stage4_composite_ms)
            results.append((statistics.median(ms), ts, rb, es))
        ms, ts, rb, es = min(results)
        best[key] = (ts, rb, es, ms)
    return best


def per_view(best: dict, compositors):
    """(tile_shape list, radix_bits list, entry_sort list) for execute_views."""
    tss, rbs, ess = [], [], []
    for comp in compositors:
        ts, rb, es, _ = best[(comp.screen_width, comp.screen_height)]
        tss.append(ts)
        rbs.append(rb)
        ess.append(es)
    return tss, rbs, ess


LAUNCH_CHOICES = {"project_threads": (256, 128, 512), "bin_blocks_per_sm": (2, 1),
                  "ranges_blocks": (1184, 592, 2368)}


def tune_launch_shape(state, scene, cages, camera, compositor, repeats: int = 3, **frame_kw):
    """Chooses the launch shape for frames like (camera, compositor) and sets
    it on `state`; returns (shape dict, median Stage 2-4 ms)."""
    best = {k: v[0] for k, v in LAUNCH_CHOICES.items()}

    def cost(shape):
        state.set_launch_shape(**shape)
        state.execute_frame_gpu(scene, cages, camera, compositor, force_stage3=True, **frame_kw)
        ms = []
        for _ in range(repeats):
            t = state.execute_frame_gpu(scene, cages, camera, compositor, force_stage3=True,
                                        profile_stages=True, **frame_kw)
            ms.append(t.stage2_project_ms + t.stage3_bin_sort_ms + t.stage4_composite_ms)
        return statistics.median(ms)

    best_ms = cost(best)
    for key, values in LAUNCH_CHOICES.items():
        for v in values[1:]:
            trial = dict(best, **{key: v})
            ms = cost(trial)
            if ms < best_ms:
                best, best_ms = trial, ms
    state.set_launch_shape(**best)
    return best, best_ms
