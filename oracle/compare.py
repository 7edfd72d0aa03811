"""ORACLE — test infrastructure only.  Comparison of GPU products with oracle products.

Grid-node decisions (status map, insideness bits) must agree exactly except at nodes whose
oracle hit lies within ``near`` of the node: those are counted and reported, not failed.
"""
from __future__ import annotations

import numpy as np


def status_ray_lims(ref, grid):
    """Oracle interval ends of the status rays, as a dict (j, k) -> array of x positions."""
    import oracle as O
    cnt, vals = O.ray_hits(ref, 0)
    x0 = grid.xmin
    dirl = (grid.xmin + (grid.nx - 1) * grid.side) - x0
    offs = np.concatenate([[0], np.cumsum(cnt.ravel())])
    return cnt, vals, offs, x0, dirl


def near_node_status(gpu_status, ref, grid, near=1e-6):
    """(#mismatching nodes, #of them that are near-node) for the status map."""
    mism = np.argwhere(gpu_status != ref.status)
    if len(mism) == 0:
        return 0, 0
    cnt, vals, offs, x0, dirl = status_ray_lims(ref, grid)
    nb = grid.ny
    n_near = 0
    for k, j, i in mism:
        r = k * nb + j
        t = vals[offs[r]:offs[r + 1]]
        lims = x0 + dirl * t
        x = grid.xmin + i * grid.side
        if len(lims) and np.min(np.abs(lims - x)) < near:
            n_near += 1
    return len(mism), n_near


def compare_surface(surf, ds, ref, rel_tol=1e-12, vert_tol=1e-9):
    """Dict of parity figures; raises AssertionError on a failure of the bar."""
    out = {}
    n_mis, n_near = near_node_status(ds.status, ref, ds.grid)
    out["status_mismatch"] = n_mis
    out["status_near_node"] = n_near
    assert n_mis == n_near, f"status map: {n_mis - n_near} mismatches away from any hit"
    out["bits_mismatch_words"] = int((surf.insideness != ref.bits).sum())
    assert out["bits_mismatch_words"] == 0, "insideness bits differ"
    assert surf.ncav == ref.ncav, f"cavity count {surf.ncav} vs {ref.ncav}"
    np.testing.assert_array_equal(np.array(ds.cavitiesSize), ref.cav_size)
    np.testing.assert_array_equal(np.array(ds.cavitiesFlag, np.int32), ref.cav_filled)
    out["volume_rel"] = abs(surf.volume - ref.volume) / abs(ref.volume)
    assert out["volume_rel"] <= rel_tol
    if surf.vertices is not None:
        np.testing.assert_array_equal(surf.vertex_edges, ref.vertex_edges)
        out["vertex_max_abs"] = float(np.abs(surf.vertices - ref.vertices).max()) if len(ref.vertices) else 0.0
        assert out["vertex_max_abs"] <= vert_tol
        np.testing.assert_array_equal(surf.triangles, ref.triangles)
        out["area_rel"] = abs(surf.area - ref.area) / abs(ref.area)
        assert out["area_rel"] <= rel_tol
    return out


def near_threshold_eps(gpu_eps, ref, grid, near=1e-6):
    """(#mismatching epsilon-map entries, #of them near a threshold of the oracle).

    Edge (node c, axis a) of a node ray is inside when its midpoint coord(c) + hside lies in an
    interval [lim1, lim2]; an entry counts as near when an oracle interval end of its ray lies
    within ``near`` of that midpoint or of coord(c) - hside (the rintp rounding of lim1)."""
    import oracle as O
    mism = np.argwhere(gpu_eps != ref.epsmap)
    if len(mism) == 0:
        return 0, 0
    mins = (grid.xmin, grid.ymin, grid.zmin)
    ns = (grid.nx, grid.ny, grid.nz)
    # axis -> (ray set, axis of m, axis of n)
    sets = {0: (0, 1, 2), 2: (4, 0, 1), 1: (5, 0, 2)}
    cache = {}
    n_near = 0
    for k, j, i, a in mism:
        s, fa, la = sets[int(a)]
        if s not in cache:
            cnt, vals = O.ray_hits(ref, s)
            cache[s] = (cnt, vals, np.concatenate([[0], np.cumsum(cnt.ravel())]))
        cnt, vals, offs = cache[s]
        idx = (i, j, k)
        m, n = idx[fa], idx[la]
        r = n * cnt.shape[1] + m
        t = vals[offs[r]:offs[r + 1]]
        x0 = mins[a]
        lims = x0 + ((x0 + (ns[a] - 1) * grid.side) - x0) * t
        c = mins[a] + idx[a] * grid.side
        if len(lims) and min(np.min(np.abs(lims - (c + grid.hside))), np.min(np.abs(lims - (c - grid.hside)))) < near:
            n_near += 1
    return len(mism), n_near
