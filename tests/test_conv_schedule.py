"""Host-side checks of the pipelined convolution's schedules (no GPU).

Restates, operation for operation, two pieces of host/issuer logic in
custom-ray-tracing-shader_b200/csrc:

- the stacked-row MMA issue of convPipeKernel (rt_conv_pipe.cu, the STACK
  branch of the issuer: segments over a ring of per-output-row accumulator
  blocks, the running block counters, the fresh block's first MMA), checked
  against what makes its results bit-identical to the tap-per-tile form:
  every output row receives taps t = 3 dy + dx with the K steps inner, in
  that order, its first MMA starts from zero, no MMA writes a block that
  holds another output row, and each block is committed once, in output
  order;
- balancedStripRows (rt_conv_tc.cuh): the strip length that minimises the
  rows the busiest block stages.
"""
import math

import pytest


def stacked_schedule(strips, nb, g2):
    """Runs the issuer's loop over strips of S output rows with a ring of nb
    blocks and g2 K steps; returns the per-output tap lists, the commit order
    and every MMA as (block, kernel row dy, output index)."""
    acc_b = 0                 # the next fresh block (accB)
    live = {}                 # block -> output index it holds
    taps = {}                 # output index -> [(t, k), ...]
    commits = []
    mmas = []
    base = 0                  # output index of the strip's row 0
    for S in strips:
        p_lo = acc_b          # block of output row jLo (pLo)
        for i in range(S + 2):
            fresh = i < S
            j_lo, j_hi = (i - 2 if i > 2 else 0), (i if i < S - 1 else S - 1)
            if fresh:
                assert acc_b not in live, 'fresh block still holds an output'
                live[acc_b] = base + i

            def segs(p, lo, hi, acc):
                n = hi - lo + 1
                run = n if n < nb - p else nb - p
                out = [(p, lo - i + 2, run, acc)]
                if run < n:
                    out.append((0, lo + run - i + 2, n - run, acc))
                return out

            rest = segs(p_lo, j_lo, j_hi, 1)
            first = list(rest)
            if fresh:
                fr = segs(acc_b, j_hi, j_hi, 0)
                first = fr if j_hi == j_lo else segs(p_lo, j_lo, j_hi - 1, 1) + fr
            assert len(first) <= 3 and len(rest) <= 2
            for dx in range(3):
                for k in range(g2):
                    for (p, beta, run, acc) in (first if dx == 0 and k == 0 else rest):
                        for q in range(run):
                            block, b = p + q, beta + q   # b: stacked weights block, dy = 2 - b
                            assert 0 <= block < nb and 0 <= b <= 2
                            out = base + (i - 2) + b
                            assert live.get(block) == out, 'MMA into a block of another output row'
                            if acc == 0:
                                assert out not in taps
                                taps[out] = []
                            taps[out].append((3 * (2 - b) + dx, k))
                            mmas.append((block, 2 - b, out))
            if i >= 2:
                out = base + i - 2
                assert live.get(p_lo) == out
                commits.append(out)
                del live[p_lo]
                p_lo = p_lo + 1 if p_lo + 1 < nb else 0
            if fresh:
                acc_b = acc_b + 1 if acc_b + 1 < nb else 0
        base += S
    return taps, commits, mmas


@pytest.mark.parametrize('nb', [3, 4, 5, 8])
@pytest.mark.parametrize('g2', [1, 2, 4])
@pytest.mark.parametrize('strips', [[1], [2], [3], [5, 5, 3], [7, 1, 4, 9], [28, 28, 13], [4] * 9, [64, 1]])
def test_stacked_issue_matches_tap_order(nb, g2, strips):
    taps, commits, mmas = stacked_schedule(strips, nb, g2)
    total = sum(strips)
    assert commits == list(range(total))
    expected = [(t, k) for t in range(9) for k in range(g2)]
    for out in range(total):
        assert taps[out] == expected, out


def test_stacked_issue_reads_each_row_once_per_tap():
    # One input row feeds at most three output rows per MMA group, and an
    # interior row uses one MMA per (dx, K step) after its first.
    taps, _, mmas = stacked_schedule([16], 4, 2)
    per_out = {}
    for block, dy, out in mmas:
        per_out.setdefault(out, set()).add(dy)
    assert all(per_out[o] == {0, 1, 2} for o in range(16))


def balanced_strip_rows(columns, h, blocks):
    best, best_cost = 1, -1
    for s in range(1, 65):
        units = columns * ((h + s - 1) // s)
        cost = (units + blocks - 1) // blocks * (s + 2)
        if best_cost < 0 or cost <= best_cost:
            best_cost, best = cost, s
        if s >= h:
            break
    return best


@pytest.mark.parametrize('columns,h,blocks', [(15, 1088, 592), (15, 1088, 1036), (8, 544, 296), (1, 68, 148),
                                              (2, 136, 148), (4, 272, 136), (32, 128, 148), (1, 3, 8)])
def test_balanced_strips_minimise_the_busiest_block(columns, h, blocks):
    s = balanced_strip_rows(columns, h, blocks)
    cost = math.ceil(columns * math.ceil(h / s) / blocks) * (s + 2)
    for t in range(1, min(h, 64) + 1):
        other = math.ceil(columns * math.ceil(h / t) / blocks) * (t + 2)
        assert cost <= other
        if other == cost:
            assert t <= s  # the longest of equals
    # The full-resolution 32-channel layer: one round of 28-row strips
    # instead of three rounds of 13 (1,260 units on 592 blocks).
    if (columns, h, blocks) == (15, 1088, 592):
        assert s == 28 and columns * math.ceil(h / s) <= blocks
