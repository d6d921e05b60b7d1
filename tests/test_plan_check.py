"""The factorization and solve plans replayed on the host (tests/plan_check.cpp):
every launch, item by item, with its kernel's arithmetic restated in FP64,
checking that each access stays in its front, that no two items of one launch
write the same entry (or one writes what another reads), and that every
contribution block still holds its front's data when read -- then D and the
solution against the oracle's up-looking LDL^T. The device runs exactly these
plans, so races, overlapping live blocks or a wrong panel grouping show here,
on a CPU. Mistakes planted in the replayed plan must be caught. CPU only."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_bin"


@pytest.fixture(scope="module")
def plan_check():
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "plancheck", "-j2"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr

    def run(variant, *args):
        return subprocess.run([str(BIN / variant), *map(str, args)], capture_output=True, text=True, timeout=900)
    return run


def _groups(out: str) -> list[tuple[int, int, int]]:
    return [tuple(map(int, m)) for m in re.findall(r"trailing 1/2/4 panels (\d+)/(\d+)/(\d+)", out)]


# (build, mode, args, the panel groupings the case must reach)
CASES = [
    ("plan_check", "cylinder", (8,), "2"),        # 2-panel groups at the production threshold
    ("plan_check", "torus", (16,), ""),           # the cut port's 2 x 2 block and its tree
    ("plan_check_g4", "cylinder", (12,), "4"),    # 4-panel groups (threshold lowered to 256 rows)
    ("plan_check", "fronts", (1, 12, 700), "2"),  # dense fronts, widths ending inside a group
    ("plan_check_g4", "fronts", (3, 10, 800), "4"),
]


@pytest.mark.parametrize("build,mode,args,reach", CASES, ids=[f"{c[0]}-{c[1]}-{c[2][0]}" for c in CASES])
def test_plan_replays_clean(plan_check, build, mode, args, reach):
    r = plan_check(build, mode, *args)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "bounds" in ln]
    assert lines and all(ln.endswith(" ok") for ln in lines), r.stdout
    for ln in lines:
        assert " bounds 0 ww 0 rw 0 stale 0 " in ln, ln
    pool = re.search(r"cb_pool (\d+) bound (\d+)", r.stdout)
    if pool:   # the CB pool within 10% of the largest total of blocks live at one level
        assert int(pool[2]) <= int(pool[1]) <= 1.1 * int(pool[2]), r.stdout
    groups = _groups(r.stdout)
    if "2" in reach:
        assert all(g[1] > 0 for g in groups), r.stdout
    if "4" in reach:
        assert all(g[2] > 0 for g in groups), r.stdout


# Edge cases of the elimination tree, each on both builds: nothing to
# factor, one unknown, no coupling at all, one dense front (wider than a
# 4-panel group), a star, disconnected cliques (many roots), a band (a path
# of supernodes, one per level), random sparsity with AMD and natural order.
PATTERNS = [("diag", 0, 1, ""), ("diag", 1, 1, ""), ("diag", 500, 1, ""), ("dense", 700, 2, ""),
            ("arrow", 2000, 1, ""), ("blocks", 3000, 5, ""), ("band", 3000, 1, "natural"),
            ("random", 4000, 7, ""), ("random", 4000, 7, "natural")]


@pytest.mark.parametrize("build", ["plan_check", "plan_check_g4"])
@pytest.mark.parametrize("shape,n,seed,order", PATTERNS, ids=[f"{p[0]}-{p[1]}-{p[3] or 'amd'}" for p in PATTERNS])
def test_edge_patterns_replay_clean(plan_check, build, shape, n, seed, order):
    r = plan_check(build, "pattern", shape, n, seed, *([order] if order else []))
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "bounds" in ln]
    assert len(lines) == 2 and all(ln.endswith(" ok") for ln in lines), r.stdout
    if shape == "dense" and build == "plan_check_g4":
        assert all(g[2] > 0 for g in _groups(r.stdout)), r.stdout   # a 4-panel group in the dense front


@pytest.mark.parametrize("mistake,caught", [
    ("overlap", r"ww [1-9]\d* rw \d+ stale [1-9]"),   # two live CBs on one another
    ("dup", r"ww [1-9]"),                             # one tile updated by two items of a launch
    ("rel", r"bounds [1-9]"),                         # a child's map repeats a row
    ("kcap", r"d_err [1-9]\.\d+e-0[1-6]"),            # a 2-panel group applied as one panel
    ("region", r"rw [1-9]"),                          # a tile reading operands nobody wrote for it
])
def test_planted_mistakes_are_caught(plan_check, mistake, caught):
    r = plan_check("plan_check", "cylinder", 8, mistake)
    assert r.returncode == 1, r.stdout + r.stderr
    assert f"planted {mistake}" in r.stdout and "FAIL" in r.stdout
    assert re.search(caught, r.stdout), r.stdout


def test_pivot_stats_threads_equal_the_sequential_walk(plan_check):
    """The per-entry factorization statistics (pivot_stats.cpp), split over
    host threads, equal the sequential walk in every field."""
    r = subprocess.run([str(BIN / "pivot_stats_check")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "DIFFERENT" not in r.stdout, r.stdout + r.stderr
