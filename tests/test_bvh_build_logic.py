"""The two steps of the GPU BVH build that replace serial code with parallel
code, checked on the CPU against the serial originals (no GPU):

* the partition. The reference calls std::partition, which libstdc++ runs as
  Hoare's two-pointer loop (bidirectional iterators). The GPU reproduces it from
  ranks: the k-th primitive left of the split that belongs on the right swaps with
  the k-th primitive right of the split, counted from the right end, that belongs
  on the left (csrc/device/bvh_gpu.cu, k_pranks / k_pswap and the warp version in
  k_small);
* the SAH sweep. The reference sweeps 16 bins per axis serially and keeps the
  first strictly cheaper plane (src/geometry/bvh.cpp:62-88). The GPU computes the
  prefix and suffix unions as scans and takes an argmin with the lowest bin
  winning ties (half_sweep / warp_best_split).
"""
import numpy as np
import pytest


def hoare_partition(items, pred):
    """libstdc++'s std::partition for bidirectional iterators, step for step."""
    a = list(items)
    first, last = 0, len(a)
    while True:
        while True:
            if first == last:
                return a, first
            if pred(a[first]):
                first += 1
            else:
                break
        last -= 1
        while True:
            if first == last:
                return a, first
            if not pred(a[last]):
                last -= 1
            else:
                break
        a[first], a[last] = a[last], a[first]
        first += 1


def rank_partition(items, pred):
    """The GPU's form: split = count of primitives that belong on the left; the
    k-th misplaced one on the left swaps with the k-th misplaced one on the right
    counted from the right end."""
    a = list(items)
    flags = [bool(pred(x)) for x in a]
    t = sum(flags)
    left_false = [i for i in range(t) if not flags[i]]
    right_true = [i for i in range(len(a) - 1, t - 1, -1) if flags[i]]
    assert len(left_false) == len(right_true)
    for i, j in zip(left_false, right_true):
        a[i], a[j] = a[j], a[i]
    return a, t


@pytest.mark.parametrize("seed", range(40))
def test_rank_partition_is_hoare_partition(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(0, 200))
    items = list(rng.permutation(n))
    bias = rng.random()
    pred_set = {x for x in items if rng.random() < bias}
    pred = lambda x: x in pred_set  # noqa: E731
    assert rank_partition(items, pred) == hoare_partition(items, pred)


def box_area(lo, hi):
    if (lo > hi).any():
        return 0.0
    e = hi - lo
    return 2.0 * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0])


def serial_sweep(blo, bhi, cnt, parent_area):
    """The reference's loop over one axis's bins (suffix, then prefix)."""
    nb = len(cnt)
    right_area, right_n = [0.0] * nb, [0] * nb
    lo, hi, c = np.full(3, np.inf), np.full(3, -np.inf), 0
    for b in range(nb - 1, 0, -1):
        lo, hi, c = np.minimum(lo, blo[b]), np.maximum(hi, bhi[b]), c + cnt[b]
        right_area[b], right_n[b] = box_area(lo, hi), c
    lo, hi, c = np.full(3, np.inf), np.full(3, -np.inf), 0
    best = (np.inf, -1, 0)
    floor = max(parent_area, 1e-30)
    for b in range(nb - 1):
        lo, hi, c = np.minimum(lo, blo[b]), np.maximum(hi, bhi[b]), c + cnt[b]
        rn = right_n[b + 1]
        if c == 0 or rn == 0:
            continue
        cost = 1.0 + (box_area(lo, hi) * c + right_area[b + 1] * rn) / floor
        if cost < best[0]:
            best = (cost, b, c)
    return best


def scan_sweep(blo, bhi, cnt, parent_area):
    """The GPU's form: inclusive prefix / suffix unions (order-free), every plane
    priced at once, then the lowest cost with the lowest bin on ties."""
    nb = len(cnt)
    plo, phi = np.minimum.accumulate(blo, axis=0), np.maximum.accumulate(bhi, axis=0)
    pn = np.cumsum(cnt)
    slo = np.minimum.accumulate(blo[::-1], axis=0)[::-1]
    shi = np.maximum.accumulate(bhi[::-1], axis=0)[::-1]
    sn = np.cumsum(cnt[::-1])[::-1]
    floor = max(parent_area, 1e-30)
    costs = []
    for b in range(nb):
        if b < nb - 1 and pn[b] != 0 and sn[b + 1] != 0:
            costs.append((1.0 + (box_area(plo[b], phi[b]) * pn[b] + box_area(slo[b + 1], shi[b + 1]) * sn[b + 1])
                          / floor, b, int(pn[b])))
        else:
            costs.append((np.inf, b, int(pn[b])))
    return min(costs, key=lambda x: (x[0], x[1]))


@pytest.mark.parametrize("seed", range(60))
def test_scan_sweep_picks_the_serial_sweeps_plane(seed):
    rng = np.random.default_rng(seed)
    nb = 16
    cnt = rng.integers(0, 4, nb) * (rng.random(nb) < 0.7)
    centre = np.sort(rng.normal(0, 1, (nb, 3)), axis=0)
    half = rng.random((nb, 3)) * 0.5
    blo, bhi = centre - half, centre + half
    blo[cnt == 0], bhi[cnt == 0] = np.inf, -np.inf  # empty bins
    if seed % 5 == 0:  # exact ties between planes
        blo[:], bhi[:] = -1.0, 1.0
    parent = box_area(blo[cnt > 0].min(axis=0), bhi[cnt > 0].max(axis=0)) if cnt.any() else 0.0
    s = serial_sweep(blo, bhi, cnt, parent)
    g = scan_sweep(blo, bhi, cnt, parent)
    if s[1] < 0:
        assert not np.isfinite(g[0])
    else:
        assert (s[0], s[1], s[2]) == (g[0], g[1], g[2])
