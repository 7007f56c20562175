"""The bench line's `gpu_launches` comes from `bench.our_launches_per_step`; the pruned search's
planning part of it is checked here against the kernel launch sites in knn_prune.cu (its
build() plus plan_items(), which build() runs for both launches)."""
import os
import re

import bench

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'nngpr_b200', 'csrc',
                   'knn_prune.cu')


def body(src, signature):
    """Source of the function whose definition starts with `signature` (up to its closing brace)."""
    start = src.index(signature)
    i = src.index('{', src.index(')', start))
    depth = 0
    for j in range(i, len(src)):
        depth += {'{': 1, '}': -1}.get(src[j], 0)
        if depth == 0:
            return src[i:j + 1]
    raise AssertionError('unbalanced braces')


def launches(code):
    return len(re.findall(r'<<<', code))


def test_planning_launches_match_the_source():
    src = open(SRC).read()
    build = body(src, 'nngp_status build(')
    plan = body(src, 'nngp_status plan_items(')
    assert 'plan_items(' in build
    planning = launches(build) + 2 * launches(plan)
    n = 434874
    # d = 3 is pruned, d = 30 is not; the seed levels are the same, so the difference is the
    # pruned search (planning, a second tile build, two searches, two merges) minus one search
    diff = bench.our_launches_per_step(n, 3, 32) - bench.our_launches_per_step(n, 30, 32)
    assert diff == planning + 1 + 2 + 2 - 1
    assert planning == 21
