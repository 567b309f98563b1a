"""Helpers to compare neighbour lists as per-particle sets."""
import numpy as np


def rows(index, elements, cap, n):
    """Per-particle sorted id arrays of a NeighborList (fixed or CSR)."""
    out = []
    index = np.asarray(index)
    elements = np.asarray(elements)
    for i in range(n):
        if cap > 0:
            r = elements[i * cap: i * cap + index[i]]
        else:
            end = index[i + 1] if i + 1 < n else elements.shape[0]
            r = elements[index[i]:end]
        out.append(np.sort(r))
    return out


def compare_capped(x, ra, rb, dist_fn, h):
    """Returns the particles whose sets differ in a way NOT explained by
    exact distance ties at the cap boundary (equal distances are ordered by
    arrival in the reference, so either member of a tie is a valid pick)."""
    bad = []
    for i, (a, b) in enumerate(zip(ra, rb)):
        if a.shape == b.shape and np.array_equal(a, b):
            continue
        if a.shape != b.shape:
            bad.append(i)
            continue
        da = {int(j): dist_fn(x[i], x[j]) for j in a}
        db = {int(j): dist_fn(x[i], x[j]) for j in b}
        only_a = set(da) - set(db)
        only_b = set(db) - set(da)
        tau = max(max(da.values()), max(db.values()))
        if not all(da[j] == tau for j in only_a) or not all(db[j] == tau for j in only_b):
            bad.append(i)
    return bad
