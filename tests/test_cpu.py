"""CPU tests: the oracle against the reference's own math (golden vectors), known answers,
an independent brute-force SES sampler, host logic of the library and its C-ABI surface."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden" / "ref_math.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_oracle_ray_sphere_matches_reference(gold, oracle_mod):
    L = oracle_mod.lib()
    inp, out = gold["sphere_in"], gold["sphere_out"]
    t = np.zeros(2)
    for row, exp in zip(inp, out):
        pa, d, c, r = (np.ascontiguousarray(row[0:3]), np.ascontiguousarray(row[3:6]),
                       np.ascontiguousarray(row[6:9]), row[9])
        ok = L.nso_ray_sphere(pa.ctypes.data, d.ctypes.data, c.ctypes.data, r, t.ctypes.data)
        assert ok == int(exp[0])
        if ok:
            assert t[0] == exp[1] and t[1] == exp[2]


def test_oracle_ray_torus_matches_reference(gold, oracle_mod):
    L = oracle_mod.lib()
    inp, out = gold["torus_in"], gold["torus_out"]
    assert len(inp) > 500
    for row, exp in zip(inp, out):
        inv = np.ascontiguousarray(row[0:9])
        tc = np.ascontiguousarray(row[9:12])
        sc = np.ascontiguousarray(row[12:15])
        probe, major, radius, panel = row[15], row[16], row[17], int(row[18])
        pa = np.ascontiguousarray(row[19:22])
        d = np.ascontiguousarray(row[22:25])
        t = np.zeros(4)
        t[:2] = row[25:27]
        n = L.nso_ray_torus(inv.ctypes.data, tc.ctypes.data, sc.ctypes.data, probe, major, radius, panel,
                            pa.ctypes.data, d.ctypes.data, t.ctypes.data)
        assert n == int(exp[0])
        np.testing.assert_array_equal(t[:n], exp[1:1 + n])


def test_jitter_generator_matches_reference(gold, native_lib):
    seed = ctypes.c_int64(1234)
    seq = [native_lib.nsg_randnum(ctypes.byref(seed)) for _ in range(64)]
    np.testing.assert_array_equal(np.array(seq), gold["randnum"])


def test_rintp_matches_reference(gold):
    np.testing.assert_array_equal(np.floor(gold["rint_in"] + 0.5), gold["rint_out"])


def test_quartic_known_roots(oracle_mod):
    L = oracle_mod.lib()
    roots = np.zeros(4)
    # (x-1)(x-2)(x-3)(x-4)
    n = L.nso_quartic(-10.0, 35.0, -50.0, 24.0, roots.ctypes.data)
    assert n == 4
    np.testing.assert_allclose(np.sort(roots), [1, 2, 3, 4], atol=1e-9)
    # (x^2+1)(x-1)(x-3): two real roots
    n = L.nso_quartic(-4.0, 4.0, -4.0, 3.0, roots.ctypes.data)
    assert n == 2
    np.testing.assert_allclose(np.sort(roots[:2]), [1, 3], atol=1e-9)
    # x^4 + 1: none
    assert L.nso_quartic(0.0, 0.0, 0.0, 1.0, roots.ctypes.data) == 0


def _surface(n, seed, scale, perfil, probe=1.4):
    atoms = generator.rsa_globule(n, seed)
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, scale, perfil)
    surf = nb.ConnollySurface(nb.ConfigFile(text=f"Probe_Radius = {probe}\n"), ds)
    surf.build()
    return atoms, ds, surf


def test_patch_builder_agrees_with_brute_force_ses(oracle_mod):
    """Status map of the oracle (fed by the host patch builder) against an independent SES
    sampler: a node is inside when a probe sphere centred there would not reach the
    solvent-accessible surface (sampled densely on the non-buried parts of the expanded spheres)."""
    from scipy.spatial import cKDTree
    atoms, ds, surf = _surface(80, 5, 2.5, 70.0)
    ref = oracle_mod.run(ds.grid, surf.patches, flags=oracle_mod.STATUS)
    g = ds.grid
    c = surf.delphi.atoms[:, :3]
    R = surf.delphi.atoms[:, 3] + 1.4
    k = np.arange(60000) + 0.5
    phi = np.arccos(1 - 2 * k / len(k))
    th = np.pi * (1 + 5 ** 0.5) * k
    u = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)
    tree = cKDTree(c)
    sas = []
    for i in range(len(c)):
        p = c[i] + R[i] * u
        ok = np.ones(len(p), bool)
        for j in tree.query_ball_point(c[i], R[i] + R.max()):
            if j != i:
                ok &= ((p - c[j]) ** 2).sum(1) >= R[j] ** 2
        sas.append(p[ok])
    sas = np.concatenate(sas)
    z, y, x = np.meshgrid(g.zmin + np.arange(g.nz) * g.side, g.ymin + np.arange(g.ny) * g.side,
                          g.xmin + np.arange(g.nx) * g.side, indexing="ij")
    q = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    d_sas, _ = cKDTree(sas).query(q)
    nbrs = tree.query_ball_point(q, R.max())
    in_union = np.array([any(((qq - c[j]) ** 2).sum() < R[j] ** 2 for j in nb_) for qq, nb_ in zip(q, nbrs)])
    brute = in_union & (d_sas >= 1.4)
    ora = (ref.status == -1).ravel()
    amb = np.abs(d_sas - 1.4) < 0.05
    assert ((ora != brute) & ~amb).sum() == 0
    assert (ora != brute).sum() < 1e-3 * len(ora)


def test_rays_are_watertight(oracle_mod):
    """Every ray of every ray set crosses the patch partition an even number of times."""
    atoms, ds, surf = _surface(327, 1, 2.0, 70.0)
    ref = oracle_mod.run(ds.grid, surf.patches)
    for s in range(4):
        cnt, _ = oracle_mod.ray_hits(ref, s)
        assert (cnt % 2).sum() == 0


def test_single_sphere_oracle_volume(oracle_mod):
    ds = nb.DelPhiShared(np.array([[0.0, 0.0, 0.0, 1.7]]), 4.0, 50.0)
    ps = nb.build_ses_patches(ds.atoms, 1.4)
    assert ps.counts[:5] == (1, 0, 0, 0, 0)
    ref = oracle_mod.run(ds.grid, ps)
    assert abs(ref.volume - 4 / 3 * np.pi * 1.7 ** 3) / (4 / 3 * np.pi * 1.7 ** 3) < 0.02
    assert abs(ref.area - 4 * np.pi * 1.7 ** 2) / (4 * np.pi * 1.7 ** 2) < 0.05


def test_two_sphere_torus_patch(oracle_mod):
    """Two atoms closer than two probe diameters: one torus, two point cells, no probe patch."""
    atoms = np.array([[0.0, 0.0, 0.0, 1.7], [3.0, 0.0, 0.0, 1.7]])
    ps = nb.build_ses_patches(atoms, 1.4)
    assert ps.counts[:5] == (2, 0, 1, 0, 0)
    # the torus: centre midway, major radius sqrt((r+p)^2 - (d/2)^2)
    tor = ps.f64[ps.i32[:, 0] == 2][0]
    np.testing.assert_allclose(tor[4:7], [1.5, 0, 0], atol=1e-12)
    np.testing.assert_allclose(tor[7], np.sqrt(3.1 ** 2 - 1.5 ** 2), rtol=1e-12)


def test_library_exports_header_symbols(native_lib):
    header = (ROOT / "include" / "nsgpu.h").read_text()
    decl = set(re.findall(r"\b(nsg_\w+)\s*\(", header))
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "nanoshaper_b200" / "lib" / "libnsgpu.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (nsg_\w+)", out))
    assert decl, "no declarations parsed"
    assert decl <= exported, f"missing: {sorted(decl - exported)}"
    for name in decl:
        getattr(native_lib, name)


def test_config_file_semantics():
    cf = nb.ConfigFile(text="# comment\nGrid_scale = 2.5 # trailing\nBuild_status_map = false\n"
                            "Surface = ses\nName = a\n  b\n\nEndConfigFile\nAfter = 1\n")
    assert cf.read("Grid_scale", 1.0) == 2.5
    assert cf.read("Build_status_map", True) is False
    assert cf.read("Surface", "x") == "ses"
    assert cf.read("Name", "") == "a\n  b"
    assert not cf.keyExists("After")
    assert cf.read("Missing", 7) == 7
    for v in ("false", "F", "no", "N", "0", "none"):
        assert nb.ConfigFile(text=f"k = {v}\n").read("k", True) is False
    assert nb.ConfigFile(text="k = yes\n").read("k", False) is True


def test_grid_build_matches_reference_formula(native_lib):
    atoms = generator.rsa_globule(50, 9)
    ds = nb.DelPhiShared(atoms, 2.0, 70.0)
    lo = (atoms[:, :3] - atoms[:, 3:]).min(0)
    hi = (atoms[:, :3] + atoms[:, 3:]).max(0)
    mid = (hi + lo) / 2
    rmax = 2 * np.max(np.abs(np.concatenate([hi - mid, lo - mid])))
    ig = int(np.floor(2.0 * 100.0 / 70.0 * rmax))
    ig += 1 - ig % 2
    assert ds.nx == ig and ds.grid.xmin == mid[0] - (ig - 1) / (2 * 2.0)


def test_generator_is_seeded():
    a = generator.rsa_globule(200, 3)
    b = generator.rsa_globule(200, 3)
    np.testing.assert_array_equal(a, b)
    from scipy.spatial import cKDTree
    d, _ = cKDTree(a[:, :3]).query(a[:, :3], k=2)
    assert d[:, 1].min() >= generator.DMIN
    assert set(np.unique(a[:, 3])) <= set(generator.RADII)


def test_cavity_label_replay_matches_oracle(native_lib, oracle_mod):
    """Host replay of the alternating seed scan over union-find regions reproduces the oracle's
    sequential flood-fill labels."""
    from scipy import ndimage
    atoms, ds, surf = _surface(327, 1, 2.0, 70.0)
    pre = oracle_mod.run(ds.grid, surf.patches, flags=oracle_mod.STATUS).status
    post = oracle_mod.run(ds.grid, surf.patches, flags=oracle_mod.STATUS | oracle_mod.CAVITIES).status
    lab, n = ndimage.label(pre == 2)
    assert n > 3
    flat = lab.ravel()
    idx = np.arange(flat.size)
    roots = np.array([idx[flat == c].min() for c in range(1, n + 1)])
    g = ds.grid
    plane = g.nx * g.ny
    desc = np.array([((g.nz - 1 - idx[flat == c] // plane) * plane + idx[flat == c] % plane).min()
                     for c in range(1, n + 1)], np.uint32)
    order = np.argsort(roots)
    labels = np.zeros(n, np.int32)
    rc = native_lib.nsg_cavity_order(n, desc[order].ctypes.data, labels.ctypes.data)
    assert rc == 0
    for pos, c in enumerate(order):
        node = roots[c]
        assert post.ravel()[node] == labels[pos]


def test_patch_gradient_chain_rule(native_lib):
    """Host chain rule from patch surface parameters to atoms (nsg_ses_chain_grad) against central
    differences of the patch parameters themselves: for a random per-patch weight vector w,
    d(sum_p w_p . theta_p(atoms)) / d(atoms) where theta is the sphere centre and radius of atom
    patches, the probe centre of facets and (tc, u, R) of tori."""
    atoms = generator.rsa_globule(60, 3)

    def theta(a):
        ps = nb.build_ses_patches(a, 1.4, 1)
        f, k = ps.f64, ps.i32[:, 0]
        th = np.zeros((ps.n, 8))
        pt = k == 0
        th[pt, :4] = f[pt, :4]
        fc = (k == 3) | (k == 4)
        th[fc, :3] = f[fc, :3]
        ed = (k == 1) | (k == 2)
        th[ed, :3] = f[ed, 4:7]
        th[ed, 3:6] = f[ed, 15:18]
        th[ed, 6] = f[ed, 7]
        return ps, th

    ps0, th0 = theta(atoms)
    w = np.random.default_rng(1).normal(size=th0.shape)
    g = ps0.chain_to_atoms(w)
    h = 1e-6
    rng = np.random.default_rng(2)
    for i in rng.choice(len(atoms), size=12, replace=False):
        for d in range(4):
            a1 = atoms.copy()
            a1[i, d] += h
            a2 = atoms.copy()
            a2[i, d] -= h
            p1, t1 = theta(a1)
            p2, t2 = theta(a2)
            assert p1.n == p2.n == ps0.n
            fd = float(((t1 - t2) * w).sum() / (2 * h))
            assert abs(fd - g[i, d]) <= 1e-6 * (abs(fd) + 1.0), (i, d, fd, g[i, d])


def test_file_writers_layouts(native_lib, tmp_path):
    """Status, cavity and mesh files follow the reference's layouts (DelPhiShared::saveStatus /
    saveCavities, Surface::saveMesh)."""
    ds = nb.DelPhiShared(np.array([[0.0, 0.0, 0.0, 1.5]]), 2.0, 50.0)
    g = ds.grid
    st = np.full((g.nz, g.ny, g.nx), 2, np.int32)
    st[1, 2, 3] = -1
    st[2, 1, 1] = 4
    st[2, 1, 2] = 4
    ds.status = st
    ds.cavitiesSize = [0.25]
    ds.cavitiesFlag = [True]
    ds.saveStatus(str(tmp_path / "run"))
    text = (tmp_path / "run.status.txt").read_text()
    blocks = text.split("\n\n")
    assert len(blocks) == g.nx + 1 and blocks[-1] == ""
    rows = blocks[3].split("\n")
    vals = [int(x) for x in rows[2].split()]
    assert len(rows) == g.ny and len(vals) == g.nz and vals[1] == -1  # i=3, j=2, k=1
    cav = (tmp_path / "cavities.txt").read_text().split("\n")
    assert cav[0] == "" and len(cav) == 3
    x1, y1, z1 = (float(v) for v in cav[1].split())
    assert abs(x1 - ds.x[1]) < 1e-6 and abs(y1 - ds.y[1]) < 1e-6 and abs(z1 - ds.z[2]) < 1e-6
    sz = (tmp_path / "cavitiesSize.txt").read_text().splitlines()
    assert sz[0] == "1.000000"
    bx, by, bz, vol, flag = sz[1].split()
    assert abs(float(bx) - 0.5 * (ds.x[1] + ds.x[2])) < 1e-6 and flag == "1" and float(vol) == 0.25
    s = nb.ConnollySurface(nb.ConfigFile(), ds)
    s.vertices = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    s.triangles = np.array([[0, 1, 2]], np.int32)
    s.saveMesh("off", True, str(tmp_path / "mesh"))
    off = (tmp_path / "mesh.off").read_text().splitlines()
    assert off[0] == "OFF" and off[1].startswith("# File created by") and off[3] == "3 1 0"
    assert off[4] == "0.000 0.000 0.000" and off[-1] == "3 2 1 0"
    assert (tmp_path / "meshtriangleAreas.txt").read_text() == "0.500000\n"
    s.saveMesh("ply", False, str(tmp_path / "mesh"))
    raw = (tmp_path / "mesh.ply").read_bytes()
    head, body = raw.split(b"end_header\n")
    assert b"element vertex 3" in head and b"element face 1" in head and len(body) == 3 * 24 + 13


def _replica_rank(rank, world, port, out):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from nanoshaper_b200 import dist as D
    pg = D.init("gloo", timeout_s=60)
    try:
        step_ms = 10.0 + 5.0 * rank  # the second replica is slower
        worst = D.max_over_ranks(pg, step_ms)
        D.barrier(pg)
        out.put((rank, worst, D.throughput(512, world, worst)))
    finally:
        D.close(pg)


def test_replica_timing_gloo_world2():
    """Two replicas over gloo: every rank sees the slowest rank's time and the whole-job
    throughput counts both ranks' structures (the bench's multi-GPU aggregation)."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, worst, thr in res:
        assert worst == 15.0
        assert abs(thr - 2 * 512 * 1000.0 / 15.0) < 1e-9


def _row_interval(cf, cl, r, mn_fd, mn_ld, side, delta, m0, m1, n):
    """The candidate kernel's row search, restated: the first pixel of the row where
    Low(m) = pa(m) >= cf - r and (dx < 0 or disc(dx)) holds and the first where
    High(m) = pa(m) <= cf + r and (dx > 0 or disc(dx)) fails, by binary search over [m0, m1]."""
    lo_fd, hi_fd, lo_ld, hi_ld, r2 = cf - r, cf + r, cl - r, cl + r, r * r
    pld = (mn_ld + float(n) * side) + delta
    if pld < lo_ld or pld > hi_ld:
        return []
    dy = cl - pld
    dy2 = dy * dy
    lo, hi = m0, m1 + 1
    while lo < hi:
        mid = (lo + hi) >> 1
        pa = (mn_fd + float(mid) * side) + delta
        dx = cf - pa
        if (not pa < lo_fd) and (dx < 0 or not dx * dx + dy2 > r2):
            hi = mid
        else:
            lo = mid + 1
    a, hi = lo, m1 + 1
    while lo < hi:
        mid = (lo + hi) >> 1
        pa = (mn_fd + float(mid) * side) + delta
        dx = cf - pa
        if (not pa > hi_fd) and (dx > 0 or not dx * dx + dy2 > r2):
            lo = mid + 1
        else:
            hi = mid
    return list(range(a, lo))


def test_candidate_row_intervals_match_pixel_test():
    """The candidate kernel replaces the reference's per-pixel bounding-box and equatorial-disc
    test (src/ConnollySurface.cpp:4469-4502) by an interval per pixel row found with two binary
    searches.  In double precision the row predicates are monotone, so the interval must hold
    exactly the pixels the per-pixel test accepts, tangent rows and pixels included."""
    import random

    def pixel_test(cf, cl, r, pfd, pld):
        if pfd < cf - r or pfd > cf + r or pld < cl - r or pld > cl + r:
            return False
        dx, dy = cf - pfd, cl - pld
        return not (dx * dx + dy * dy > r * r)

    rng = random.Random(11)
    rows = 0
    for _ in range(3000):
        side = rng.choice([0.5, 1.0 / 3.0, 0.25, 1.0 / 2.2])
        mn_fd, mn_ld = rng.uniform(-50, 50), rng.uniform(-50, 50)
        delta = rng.choice([0.0, 1e-10 - side / 2])
        mc, nc = rng.randint(0, 40), rng.randint(0, 40)
        kind = rng.random()
        if kind < 0.4:  # centre on a pixel, radius a multiple of the spacing: exact tangencies
            cf, cl = (mn_fd + float(mc) * side) + delta, (mn_ld + float(nc) * side) + delta
            r = side * rng.randint(1, 10)
        else:
            cf, cl = mn_fd + rng.uniform(0, 40) * side, mn_ld + rng.uniform(0, 40) * side
            r = rng.uniform(0.1, 6.0)
        m0 = max(0, int(round((cf - r - mn_fd) / side)) - rng.randint(0, 2))
        m1 = int(round((cf + r - mn_fd) / side)) + rng.randint(-1, 2)
        n0 = max(0, int(round((cl - r - mn_ld) / side)) - 1)
        n1 = int(round((cl + r - mn_ld) / side)) + 1
        for n in range(n0, n1 + 1):
            want = [m for m in range(m0, m1 + 1)
                    if pixel_test(cf, cl, r, (mn_fd + float(m) * side) + delta, (mn_ld + float(n) * side) + delta)]
            assert _row_interval(cf, cl, r, mn_fd, mn_ld, side, delta, m0, m1, n) == want
            rows += 1
    assert rows > 10000


def test_pipelined_chunk_bounds():
    """Chunks of an ensemble cover every structure once, in order, with no empty chunk, and the
    first is about half the size of the others."""
    from nanoshaper_b200.pipelined import chunk_bounds
    for n in range(1, 80):
        for k in range(1, 10):
            b = chunk_bounds(n, k)
            assert b[0] == 0 and b[-1] == n and len(b) - 1 <= min(n, k)
            assert np.all(np.diff(b) > 0)
    b = chunk_bounds(512, 6)
    sizes = np.diff(b)
    assert len(sizes) == 6 and abs(sizes[0] - sizes[1] / 2) <= 1 and sizes[1:].max() - sizes[1:].min() <= 1


def test_bench_reference_arm_contract():
    """`bench.py --impl reference` (the oracle port on the host cores) prints one JSON line with
    the driver's keys, on the small ensemble."""
    import json
    import sys
    root = Path(__file__).resolve().parents[1]
    res = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--workload", "ensemble_64",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=root)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads([ln for ln in res.stdout.splitlines() if ln.startswith("{")][-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_mesh_normals_and_normal_formats(native_lib, tmp_path):
    """Triangle-averaged vertex normals (approximateNormals without analytic normals), nearest atoms
    (vdwAccessible) and the OFF+N, OFF+A, OFF+N+A and MSMS writers (Surface::saveMesh)."""
    v = np.array([[1.0, 0, 0], [-1.0, 0, 0], [0, 1.0, 0], [0, -1.0, 0], [0, 0, 1.0], [0, 0, -1.0]])
    # octahedron, counter-clockwise seen from outside
    t = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]], np.int32)
    ds = nb.DelPhiShared(np.array([[0.0, 0.0, 0.0, 1.5]]), 2.0, 50.0)
    s = nb.ConnollySurface(nb.ConfigFile(), ds)
    s.vertices, s.triangles = v, t
    n = s.approximateNormals()
    # numpy restatement: sum of the unnormalised plane normals (p2 - p1) x (p3 - p1) per vertex
    ref = np.zeros_like(v)
    for a, b, c in t:
        w = np.cross(v[b] - v[a], v[c] - v[a])
        ref[a] += w
        ref[b] += w
        ref[c] += w
    ref /= np.linalg.norm(ref, axis=1, keepdims=True)
    assert np.allclose(n, ref, atol=1e-15) and np.allclose(n, v, atol=1e-15)
    s.saveMesh("off_n", False, str(tmp_path / "m"))
    off = (tmp_path / "m.off").read_text().splitlines()
    assert off[0] == "OFF+N" and off[3] == "6 8 0"
    assert off[4] == "1.000 0.000 0.000 1.000 0.000 0.000" and off[-1] == "3 0 3 5"
    assert len((tmp_path / "mtriangleAreas.txt").read_text().splitlines()) == 8
    s.delphi.atoms = np.array([[2.0, 0, 0, 1.5], [0, 0, 2.5, 1.0], [-2.0, 0.1, 0, 1.7]])
    va = s.vertexAtoms()
    pd = ((v[:, None, :] - s.delphi.atoms[None, :, :3]) ** 2).sum(-1) - s.delphi.atoms[None, :, 3] ** 2
    assert np.array_equal(va, np.argmin(pd, axis=1))
    s.saveMesh("off_n_a", False, str(tmp_path / "a"))
    offa = (tmp_path / "a.off").read_text().splitlines()
    assert offa[0] == "OFF+N+A" and offa[4] == "1.000 0.000 0.000 1.000 0.000 0.000 %d" % va[0]
    s.saveMesh("off_a", False, str(tmp_path / "b"))
    assert (tmp_path / "b.off").read_text().splitlines()[4] == "1.000 0.000 0.000 %d" % va[0]
    s.saveMesh("msms", False, str(tmp_path / "c"))
    assert (tmp_path / "c.vert").read_text().splitlines()[3].split()[7] == str(va[0] + 1)
    s.saveMesh("msms_no_a", True, str(tmp_path / "m"))
    face = (tmp_path / "m.face").read_text().splitlines()
    assert face[0].startswith("# File created by") and face[1] == "#faces" and face[2] == "8"
    assert face[3].split() == ["5", "3", "1", "1", "1"] and len(face) == 11  # reverted, 1-based
    vert = (tmp_path / "m.vert").read_text().splitlines()
    assert vert[1] == "#vertex" and vert[2] == "6" and len(vert) == 9
    cols = vert[3].split()
    assert len(cols) == 9 and cols[:6] == ["1.000", "0.000", "0.000", "1.000", "0.000", "0.000"] and cols[6:] == ["0", "1", "0"]
    assert vert[3] == "%9.3f %9.3f %9.3f %9.3f %9.3f %9.3f %7d %7d %2d " % (1, 0, 0, 1, 0, 0, 0, 1, 0)


def test_vertex_atoms_match_brute_force(native_lib):
    """The nearest-atom search (shells of grid cells) equals the brute-force least power distance
    on random globules, vertices inside, on and far outside the atoms' box."""
    rng = np.random.default_rng(4)
    L = nb._native.lib()
    for trial in range(20):
        n = int(rng.integers(1, 300))
        atoms = np.concatenate([rng.uniform(-15, 15, (n, 3)), rng.uniform(1.0, 2.2, (n, 1))], axis=1)
        verts = rng.uniform(-25, 25, (500, 3))
        verts[:50] = atoms[rng.integers(0, n, 50), :3] + rng.normal(0, 0.5, (50, 3))
        out = np.zeros(len(verts), np.int32)
        assert L.nsg_vertex_atoms(verts.ctypes.data, len(verts), atoms.ctypes.data, n, out.ctypes.data) == 0
        pd = ((verts[:, None, :] - atoms[None, :, :3]) ** 2).sum(-1) - atoms[None, :, 3] ** 2
        assert np.array_equal(out, np.argmin(pd, axis=1))


def test_pqr_reader_and_facade_input(native_lib, tmp_path):
    """pqr files are read as DelPhiShared::loadAtoms reads them: ATOM / HETATM records with 10 or
    11 fields, other records skipped, zero-radius atoms dropped, a malformed record an error; the
    facade takes an xyzr or pqr file, or XYZR_FileName from the configuration."""
    pqr = tmp_path / "mol.pqr"
    pqr.write_text("REMARK  generated\n"
                   "ATOM      1  N   MET A   1      1.000   2.000   3.000  -0.30 1.8500\n"
                   "ATOM      2  H   MET A   1      1.500   2.500   3.500   0.30 0.0000\n"
                   "HETATM    3  O   HOH     2     -4.250   0.000  10.500  -0.80 1.5200\n"
                   "\n"
                   "TER\n"
                   "END\n")
    a = nb.read_pqr(pqr)
    assert a.shape == (2, 4)
    assert np.array_equal(a, [[1.0, 2.0, 3.0, 1.85], [-4.25, 0.0, 10.5, 1.52]])
    assert np.array_equal(nb.read_atoms(pqr), a)
    bad = tmp_path / "bad.pqr"
    bad.write_text("ATOM      1  N   MET A   1      1.000   2.000   3.000  -0.30\n")
    with pytest.raises(nb._native.NativeError):
        nb.read_pqr(bad)
    xyzr = tmp_path / "mol.xyzr"
    xyzr.write_text("1.0 2.0 3.0 1.85\n-4.25 0.0 10.5 1.52\n")
    assert np.array_equal(nb.read_atoms(xyzr), a)
    ns = nb.NanoShaper(str(pqr))
    assert np.array_equal(ns.ds.atoms, a)
    cf = nb.ConfigFile()
    cf.add("XYZR_FileName", str(xyzr))
    assert np.array_equal(nb.NanoShaper(config=cf).ds.atoms, a)


def test_mc_case_table_matches_reference_tritable():
    """The marching-cubes case table (csrc/mc_cases.h) equals the reference's triTable
    (src/tools.h:181, extracted into tests/golden/fixtures/mc_tritable.npy) on all 256 cases."""
    root = Path(__file__).resolve().parent.parent
    text = (root / "nanoshaper_b200" / "csrc" / "mc_cases.h").read_text()
    body = text[text.index("kNsMcCases[256]"):]
    cases = re.findall(r'"([0-9a-b]*)"', body)
    assert len(cases) == 256
    ref = np.load(root / "tests" / "golden" / "fixtures" / "mc_tritable.npy")
    for c, s in enumerate(cases):
        ours = [int(ch, 16) for ch in s]
        theirs = [int(v) for v in ref[c] if v >= 0]
        assert ours == theirs, f"case {c}: {ours} vs {theirs}"


def test_reference_fixture_config_parses(native_lib):
    """The reference's own 1crn SES configuration, read through ConfigFile, drives the facade: the
    atoms come from its XYZR_FileName (resolved beside the .prm), the grid from Grid_scale and
    Grid_perfil."""
    fx = Path(__file__).resolve().parent / "golden" / "fixtures"
    cf = nb.ConfigFile(fx / "1crn_ses_conf.prm")
    assert cf.read("Surface", "", str).strip() == "ses"
    assert cf.read("Grid_perfil", 0.0, float) == 90.0
    assert cf.read("Compute_Vertex_Normals", False, bool) is True
    ns = nb.NanoShaper(config=cf)
    assert len(ns.ds.atoms) == 327
    assert ns.scale == 2.0 and ns.perfil == 90.0
    ref_atoms = nb.read_xyzr(fx / "1crn.xyzr")
    np.testing.assert_array_equal(ns.ds.atoms, ref_atoms)


def test_skin_predicates_signs(native_lib):
    """Orientation and orthosphere-conflict predicates of the skin builder's triangulation on
    integer points: the unit tetrahedron is positively oriented, a point inside its circumsphere
    conflicts, a far point does not, and a point whose negative weight exceeds its power distance
    to the orthosphere does not."""
    import ctypes
    from nanoshaper_b200 import _native as N
    L = native_lib

    def pred(p):
        p = np.ascontiguousarray(p, np.int64)
        o, c = ctypes.c_int(), ctypes.c_int()
        assert L.nsg_skin_predicates(N.ptr(p), ctypes.byref(o), ctypes.byref(c)) == 0
        return o.value, c.value

    base = [[0, 0, 0, 0], [1000, 0, 0, 0], [0, 1000, 0, 0], [0, 0, 1000, 0]]
    assert pred(base + [[250, 250, 250, 0]]) == (1, 1)
    assert pred(base + [[3000, 3000, 3000, 0]]) == (1, 0)
    assert pred(base + [[250, 250, 250, -10 ** 7]]) == (1, 0)
    swapped = [base[1], base[0], base[2], base[3]]
    assert pred(swapped + [[250, 250, 250, 0]])[0] == -1
    # large coordinates: exact at the 2^33 bound of the snapped grid
    big = np.array(base + [[250, 250, 250, 0]], np.int64)
    big[:, :3] *= 2 ** 23
    big[:, 3] *= 2 ** 46
    assert pred(big) == (1, 1)


def _skin(atoms, scale, perfil, s=0.45):
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, scale, perfil)
    cf = nb.ConfigFile(text=f"Surface = skin\nSkin_Surface_Parameter = {s}\nAccurate_Triangulation = true\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    return ds, surf


def test_skin_single_atom_is_its_sphere(native_lib, oracle_mod):
    """One atom: a single Del0 cell without planes whose quadric is the atom sphere; the ray-cast
    volume tends to 4/3 pi r^3."""
    atoms = np.array([[0.0, 0.0, 0.0, 1.7]])
    ds, surf = _skin(atoms, 6.0, 50.0)
    p = surf.patches
    assert p.n == 1 and p.i32[0, 0] == 5 and p.i32[0, 2] == 0
    r = oracle_mod.run(ds.grid, p, flags=oracle_mod.STATUS)
    exact = 4.0 / 3.0 * np.pi * 1.7 ** 3
    assert abs(r.volume - exact) / exact < 0.01


def test_skin_cells_tile_space_and_match_the_ray_cast(native_lib, oracle_mod):
    """The mixed cells of a 30-atom globule: no grid node lies in two cells; at every node inside a
    cell the sign of the cell's quadric (inside: < 0, > 0 for reduced tetrahedra) equals the
    oracle's ray-cast status; every ray of the four ray sets has an even hit count."""
    atoms = generator.rsa_globule(30, 1)
    ds, surf = _skin(atoms, 3.0, 60.0)
    p = surf.patches
    r = oracle_mod.run(ds.grid, p, flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION)
    for s in range(4):
        cnt, _ = oracle_mod.ray_hits(r, s)
        assert int((cnt % 2).sum()) == 0, f"ray set {s}: rays with odd hit counts"
    zz, yy, xx = np.meshgrid(ds.z, ds.y, ds.x, indexing="ij")
    X = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    status_in = r.status.ravel() == -1
    cell_in = np.zeros(len(X), bool)
    covered = np.zeros(len(X), np.int32)
    for i in range(p.n):
        kind, first, cnt = p.i32[i, :3]
        f = p.f64[i]
        idx = np.nonzero(np.all((X >= f[14:17]) & (X <= f[17:20]), axis=1))[0]
        if len(idx) == 0:
            continue
        Y = X[idx]
        ok = np.ones(len(idx), bool)
        for q in range(first, first + cnt):
            ok &= (Y @ p.pool[q, :3] + p.pool[q, 3]) <= 0
        idx, Y = idx[ok], Y[ok]
        q11, q22, q33, q44, q12, q23, q34, q13, q24, q14 = f[4:14]
        x, y, z = Y[:, 0], Y[:, 1], Y[:, 2]
        v = (q11 * x * x + q22 * y * y + q33 * z * z + 2 * q12 * x * y + 2 * q23 * y * z + 2 * q13 * x * z +
             2 * q14 * x + 2 * q24 * y + 2 * q34 * z + q44)
        covered[idx] += 1
        cell_in[idx] = v > 0 if kind == 8 else v < 0
    assert covered.max() <= 1
    cov = covered > 0
    assert cov.sum() > 0.2 * len(X)
    assert np.array_equal(cell_in[cov], status_in[cov])


def test_skin_reference_fixture_1crn_is_watertight(native_lib, oracle_mod):
    """The reference's 1crn skin fixture (its .prm through ConfigFile): the mixed complex ray casts
    to an even hit count on every ray of the four ray sets."""
    fx = Path(__file__).resolve().parent / "golden" / "fixtures"
    cf = nb.ConfigFile(fx / "1crn_skin_conf.prm")
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    assert ns.surf.name == "skin" and ns.surf.getShrinking() == 0.45
    ns.buildAnalyticalSurface()
    p = ns.surf.patches
    assert p.counts[5] == 327
    r = oracle_mod.run(ns.ds.grid, p, flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION)
    for s in range(4):
        cnt, _ = oracle_mod.ray_hits(r, s)
        assert int((cnt % 2).sum()) == 0
    assert r.volume > 0


def test_blobby_oracle_mesh_is_closed_and_matches_field(native_lib, oracle_mod):
    """The oracle's blobby mesh (field, marching cubes, smoothing, OFF round trip) of a 60-atom
    globule: every vertex is used and finite, the coordinates carry the OFF text's 3 decimals, every
    ray of the four ray sets has an even hit count, and the ray-cast volume is within 3% of the
    field's inside-node count times side^3."""
    atoms = generator.rsa_globule(60, 2)
    ds = nb.DelPhiShared(atoms, 3.0, 70.0)
    v, keys, t = oracle_mod.blobby_mesh(ds.grid, ds.atoms, -2.5, True)
    used = np.zeros(len(v), bool)
    used[t.ravel()] = True
    assert used.all() and np.isfinite(v).all()
    assert np.allclose(v, np.round(v.astype(np.float64), 3), atol=1e-5)
    r = oracle_mod.run(ds.grid, oracle_mod.TrianglePatches(v, t),
                       flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION)
    for s in range(4):
        cnt, _ = oracle_mod.ray_hits(r, s)
        assert int((cnt % 2).sum()) == 0
    g = ds.grid
    xs = g.xmin + np.arange(g.nx) * g.side - g.hside
    ys = g.ymin + np.arange(g.ny) * g.side - g.hside
    zs = g.zmin + np.arange(g.nz) * g.side - g.hside
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    f = np.zeros(X.shape)
    for a in ds.atoms:
        d2 = (X - a[0]) ** 2 + (Y - a[1]) ** 2 + (Z - a[2]) ** 2
        f += np.exp(-2.5 * (d2 / a[3] ** 2 - 1))
    vol_nodes = (f > 1.0).sum() * g.side ** 3
    assert abs(r.volume - vol_nodes) <= 0.03 * vol_nodes


def test_oracle_epsilon_map_rules(oracle_mod):
    """Epsilon map of the oracle against the rule it restates, checked from the oracle's own ray
    hits: the edge from node c along an axis is inside exactly when its midpoint coord(c) + hside
    lies in an interval of its node ray (src/Surface.cpp:6645-6680, 6786-6795, 6887-6896); the ideb
    map is the complement of the status map's inside nodes; the boundary grid points are the nodes
    whose six edge codes differ (src/Surface.cpp:1488-1546), all external with one inside code."""
    atoms, ds, surf = _surface(60, 3, 2.0, 70.0)
    O = oracle_mod
    ref = O.run(ds.grid, surf.patches, flags=O.STATUS | O.EPSMAP | O.BGP)
    g = ds.grid
    eps = ref.epsmap
    assert set(np.unique(eps).tolist()) == {0, 5}
    mins = (g.xmin, g.ymin, g.zmin)
    ns = (g.nx, g.ny, g.nz)
    n_checked = n_tie = 0
    for axis, s, fa, la in ((0, 0, 1, 2), (2, 4, 0, 1), (1, 5, 0, 2)):
        cnt, vals = O.ray_hits(ref, s)
        offs = np.concatenate([[0], np.cumsum(cnt.ravel())])
        mid = mins[axis] + np.arange(ns[axis]) * g.side + g.hside
        x0 = mins[axis]
        dirl = (x0 + (ns[axis] - 1) * g.side) - x0
        for n in range(cnt.shape[0]):
            for m in range(cnt.shape[1]):
                r = n * cnt.shape[1] + m
                t = vals[offs[r]:offs[r + 1]]
                want = np.zeros(ns[axis], bool)
                near = np.zeros(ns[axis], bool)
                if len(t) and len(t) % 2 == 0:
                    for q in range(0, len(t), 2):
                        if abs(t[q + 1] - t[q]) < 1e-8:
                            continue
                        l1, l2 = x0 + dirl * t[q], x0 + dirl * t[q + 1]
                        want |= (mid >= l1) & (mid <= l2)
                        near |= (np.abs(mid - l1) < 1e-9) | (np.abs(mid - l2) < 1e-9)
                idx = [0, 0, 0]
                idx[fa], idx[la] = m, n
                line = [slice(None)] * 3
                line[2 - fa], line[2 - la] = m, n  # eps is indexed [k, j, i]
                got = eps[tuple(line) + (axis,)] == 5
                ok = (got == want) | near
                assert ok.all(), f"axis {axis} ray (m={m}, n={n}): {np.flatnonzero(~ok)}"
                n_checked += len(got)
                n_tie += int(near.sum())
    assert n_checked == 3 * g.nx * g.ny * g.nz and n_tie < 10
    # ideb: the complement of the inside nodes (no cavity filled here)
    np.testing.assert_array_equal(ref.idebmap, ref.status != -1)
    # boundary grid points: the nodes whose six edge codes differ, in (z, y, x) scan order
    e = eps
    c0 = e[1:, 1:, 1:, 0]
    diff = (c0 != e[1:, 1:, 1:, 1]) | (c0 != e[1:, 1:, 1:, 2]) | (c0 != e[1:, 1:, :-1, 0]) | \
           (c0 != e[1:, :-1, 1:, 1]) | (c0 != e[:-1, 1:, 1:, 2])
    kji = np.argwhere(diff) + 1
    np.testing.assert_array_equal(ref.ibgp, kji[:, ::-1])
    assert (ref.bgp_type == 1).all() and ref.nbgp > 0


def test_oracle_bgp_projection_single_atom(oracle_mod):
    """One atom: the SES is its sphere, and every boundary grid point projects radially onto it."""
    O = oracle_mod
    ds = nb.DelPhiShared(np.array([[0.3, -0.2, 0.1, 1.7]]), 4.0, 50.0)
    ps = nb.build_ses_patches(ds.atoms, 1.4)
    ref = O.run(ds.grid, ps, flags=O.STATUS | O.EPSMAP | O.BGP)
    assert ref.nbgp > 0 and (ref.bgp_flag == 0).all()
    c = ds.atoms[0, :3]
    y = np.stack([ds.x[ref.ibgp[:, 0]], ds.y[ref.ibgp[:, 1]], ds.z[ref.ibgp[:, 2]]], 1)
    np.testing.assert_allclose(np.linalg.norm(ref.scspos - c, axis=1), 1.7, atol=1e-12)
    u = (y - c) / np.linalg.norm(y - c, axis=1)[:, None]
    np.testing.assert_allclose(ref.scspos, c + 1.7 * u, atol=1e-12)
    assert not ref.scsnor.any()
    # every point lies within one grid diagonal of the sphere
    assert np.abs(np.linalg.norm(y - c, axis=1) - 1.7).max() <= np.sqrt(3) * ds.side


def test_oracle_operation_counters_are_consistent(oracle_mod):
    """The oracle's branch counters (the bench's operation model) add up: every torus candidate
    with a clipping-sphere hit leaves the quartic's head with 0, 2 or 4 roots, every quartic with
    roots takes exactly one resolvent branch, and the model's totals follow the counts."""
    import ctypes
    atoms, ds, surf = _surface(300, 1, 2.0, 70.0)
    O = oracle_mod
    p = surf.patches
    L = O.lib()
    h = L.nso_run_ex(ctypes.byref(ds.grid), p.n, p.f64.ctypes.data, p.i32.ctypes.data, p.pool.ctypes.data,
                     p.pool_flag.ctypes.data, p.probe, O.STATUS | O.ACCURATE_TRIANGULATION, 0.0, 4, 50)
    c = O.op_counts(h)
    L.nso_free(h)
    assert c["torus_cand"] > 0 and c["sphere_cand"] > 0
    assert c["quartic_none"] + c["quartic_2"] + c["quartic_4"] == c["torus_cand"] - c["torus_no_sphere"]
    branches = c["cubic_small_c"] + c["cubic_ratio_sqrt"] + c["cubic_ratio_eps"] + c["cubic_cbrt"] + c["cubic_acos"]
    assert branches == c["quartic_2"] + c["quartic_4"]
    assert c["root_in"] <= c["root_test"]
    m = O.op_model(c)
    assert m["flops"] >= 15 * (c["torus_cand"] + c["sphere_cand"])
    assert m["cbrt"] == 2 * c["cubic_cbrt"] and m["acos"] == c["cubic_acos"]


def test_cxx_surface_binding_compiles_and_links(native_lib, tmp_path):
    """The reference-side Surface subclass of the integration notes (tests/cxx/gpu_ses_surface.h)
    compiles against a stand-in of the reference's interface and links against libnsgpu.so."""
    import shutil
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    from nanoshaper_b200 import build as B
    out = tmp_path / "gss"
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           "-I", str(ROOT / "tests" / "cxx" / "reference_stub"), "-I", str(ROOT / "tests" / "cxx"),
           str(ROOT / "tests" / "cxx" / "gpu_ses_surface_main.cpp"), "-L", str(B.LIB_DIR), "-lnsgpu", "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_oracle_cavity_atoms_against_loops(oracle_mod):
    """The oracle's vectorised cavity atoms (getCavitiesAtomsWithBilevelStatusMap) equal a direct
    loop transcription of the reference's scan: boundary nodes of each cavity, the 27 atom-grid
    cells in shift_map order, atoms in cell order, strict power-distance minimum, -1 for empty
    neighbourhoods.  Synthetic status map: two box cavities and one cavity touching the grid edge
    (its nodes on the grid boundary see TEMPORARY_OUT outside)."""
    atoms, ds, surf = _surface(120, 3, 2.0, 70.0)
    g = ds.grid
    O = oracle_mod
    st = np.full((g.nz, g.ny, g.nx), -1, np.int32)
    st[:2, :, :] = 3
    st[5:9, 6:10, 7:12] = 4
    st[12:15, 4:7, 9:11] = 5
    st[g.nz - 3:, g.ny - 4:, : 3] = 6
    ncav = 3
    got = O.cavity_atoms(g, st, ncav, ds.atoms)
    ggrid, gmin, gscale, cells = O.atom_grid(g, ds.atoms)
    want = [set() for _ in range(ncav)]
    nz, ny, nx = st.shape

    def at(i, j, k):
        return st[k, j, i] if 0 <= i < nx and 0 <= j < ny and 0 <= k < nz else 2

    for k, j, i in zip(*[v.tolist() for v in np.nonzero(st >= 4)]):
        s = st[k, j, i]
        if all(at(*q) == s for q in ((i + 1, j, k), (i - 1, j, k), (i, j + 1, k), (i, j - 1, k),
                                     (i, j, k + 1), (i, j, k - 1))):
            continue
        p = (g.xmin + i * g.side, g.ymin + j * g.side, g.zmin + k * g.side)
        c = [int(np.floor((p[d] - gmin[d]) * gscale + 0.5)) for d in range(3)]
        best, first = np.inf, -1
        for sx, sy, sz in O.SHIFT27:
            cx, cy, cz = c[0] + sx, c[1] + sy, c[2] + sz
            if not (0 <= cx < ggrid and 0 <= cy < ggrid and 0 <= cz < ggrid):
                continue
            for a in cells.get((cz * ggrid + cy) * ggrid + cx, []):
                x = ds.atoms[a]
                d = (x[0] - p[0]) * (x[0] - p[0]) + (x[1] - p[1]) * (x[1] - p[1]) + (x[2] - p[2]) * (x[2] - p[2])
                d -= x[3] * x[3]
                if d < best:
                    best, first = d, a
        want[s - 4].add(first)
    assert got == [sorted(w) for w in want]
    assert all(len(x) > 0 for x in got)


def test_write_cavity_atoms_layout(native_lib, tmp_path):
    """cavAtomsSerials.txt: one line per cavity, "%d " per atom serial (index + 1, or the given
    serial), -1 written as 0, skipped cavities left out (DelPhiShared::saveCavities)."""
    from nanoshaper_b200 import _native as N
    off = np.array([0, 3, 3, 5], np.int32)
    lst = np.array([-1, 4, 9, 0, 2], np.int32)
    p = tmp_path / "cavAtomsSerials.txt"
    N.check(N.lib().nsg_write_cavity_atoms(str(p).encode(), 3, N.ptr(off), N.ptr(lst), None, 10, None), "write")
    assert p.read_text() == "0 5 10 \n\n1 3 \n"
    serials = np.arange(100, 110, dtype=np.int32)
    skip = np.array([0, 1, 0], np.int32)
    N.check(N.lib().nsg_write_cavity_atoms(str(p).encode(), 3, N.ptr(off), N.ptr(lst), N.ptr(serials), 10,
                                           N.ptr(skip)), "write")
    assert p.read_text() == "0 104 109 \n100 102 \n"


def _box_grid(n: int, scale: float):
    from nanoshaper_b200 import _native as N
    g = N.NsGrid()
    g.nx = g.ny = g.nz = n
    g.xmin = g.ymin = g.zmin = -3.0
    g.xmax = g.ymax = g.zmax = -3.0 + (n - 1) / scale
    g.scale, g.side, g.hside = scale, 1.0 / scale, 0.5 / scale
    return g


def _shape_fixed_point(g, lab, filled, r, mod):
    """The device formulation of the water-shape filter, restated in Python: supports read the
    removed set of the pass before for the earlier cavities, passes repeat until the removed set
    settles; then the status codes."""
    nz, ny, nx = lab.shape
    X = [g.xmin + i * g.side for i in range(nx)]

    def box(q, n):
        x = g.xmin + q * g.side
        lo = int(np.floor(((x - r) - g.xmin) * g.scale + 0.5))
        hi = int(np.floor(((x + r) - g.xmin) * g.scale + 0.5))
        return min(max(lo, 0), n - 1), min(max(hi, 0), n - 1)

    def sphere(k, j, i):
        (z0, z1), (y0, y1), (x0, x1) = box(k, nz), box(j, ny), box(i, nx)
        for z in range(z0, z1 + 1):
            for y in range(y0, y1 + 1):
                for x in range(x0, x1 + 1):
                    a, b, c = X[x] - X[i], X[y] - X[j], X[z] - X[k]
                    if a * a + b * b + c * c <= r * r:
                        yield z, y, x

    nodes = [tuple(v) for v in np.argwhere(lab >= 4) if not filled[lab[tuple(v)] - 4]]
    prev = None
    for t in range(len(filled) + 1):
        sup = {v for v in nodes if all(lab[u] == lab[v] or (prev is not None and u in prev and 4 <= lab[u] < lab[v])
                                       for u in sphere(*v))}
        own, later = set(), set()
        for v in sup:
            for u in sphere(*v):
                (own if lab[u] == lab[v] else later).add(u)
        removed = {v for v in nodes if v not in own}
        if mod or (t > 0 and removed == prev):
            break
        prev = removed
    st = lab.copy()
    for v in nodes:
        L = lab[v]
        st[v] = -L if v in sup else (L if v not in removed else (-1 if mod else (-2 if v in later else -3)))
    return st, removed


def test_oracle_shape_filter_known_cube(oracle_mod):
    """An 8^3 block cavity at scale 1 with a 1.4 A probe: the probe sphere is a node and its six
    face neighbours, so the 6^3 interior nodes are supports and the 12 edges (with the corners,
    80 nodes) are removed; the cavity stays open."""
    g = _box_grid(14, 1.0)
    lab = np.full((14, 14, 14), -1, np.int32)
    lab[:2] = 3
    lab[3:11, 3:11, 3:11] = 4
    st, fl, _b, _e, _d, nrem = oracle_mod.shape_filter(g, lab, 1, [0], probe=1.4)
    assert nrem == 80 and fl.tolist() == [0]
    assert (st == -4).sum() == 216 and (st == 4).sum() == 512 - 216 - 80 and (st == -3).sum() == 80
    st2, fl2, *_rest, nrem2 = oracle_mod.shape_filter(g, lab, 1, [0], probe=1.4, mod_status=True)
    assert nrem2 == 80 and (st2 == -1).sum() == (lab == -1).sum() + 80


def test_oracle_shape_filter_matches_fixed_point(oracle_mod):
    """The oracle's cavity-by-cavity loops equal the device's fixed-point formulation on touching
    cavities with ragged walls (the removed nodes of an earlier cavity count for a later one when
    the status map is kept), a thin cavity removed completely (flagged filled) and a filled one
    (skipped)."""
    g = _box_grid(26, 2.0)
    rng = np.random.default_rng(7)
    lab = np.full((26, 26, 26), -1, np.int32)
    lab[:2] = 3
    lab[3:13, 3:20, 3:20] = 4
    lab[13:22, 3:20, 3:20] = 5
    lab[6:9, 22:24, 4:20] = 6           # two nodes thick: no probe sphere fits
    lab[18:22, 21:24, 21:24] = 7        # filled by the volume threshold
    noise = rng.random(lab.shape) < 0.04
    lab[noise & (lab >= 4) & (lab <= 5)] = -1
    filled = [0, 0, 0, 1]
    cross = False
    for mod in (False, True):
        st, fl, _b, _e, _d, nrem = oracle_mod.shape_filter(g, lab, 4, filled, probe=1.4, mod_status=mod)
        want, removed = _shape_fixed_point(g, lab, filled, 1.4, mod)
        np.testing.assert_array_equal(st, want)
        assert nrem == len(removed)
        assert fl.tolist()[2:] == [1, 1] and fl.tolist()[:2] == [0, 0]
        if not mod:
            own_only, _ = _shape_fixed_point(g, lab, filled, 1.4, True)
            cross = bool(((want == -4 - 1) != (own_only == -4 - 1)).any())
    assert cross, "the case should exercise removed nodes of cavity 4 inside supports of cavity 5"


def test_oracle_pocket_difference_known(oracle_mod):
    """Pocket difference on synthetic maps at scale 1: a solid block for the fat surface and, for
    the small one, the same block with a 7^3 pit and a 2^3 pit.  The 7^3 difference keeps its
    5^3 core and faces after the 1.4 A water filter (the 68 edge and corner nodes go), one pocket
    of 275 A^3; the 2^3 pit holds no water probe and vanishes.  A filling threshold of 300 A^3
    fills it and clears its insideness bits."""
    g = _box_grid(30, 1.0)
    st1 = np.full((30, 30, 30), 3, np.int32)
    st1[2:28, 2:28, 2:28] = -1
    st2 = st1.copy()
    st2[4:11, 5:12, 5:12] = 2
    st2[15:17, 15:17, 15:17] = 2
    words = ((30 + 31) >> 5) * 30 * 30
    bits = np.zeros(words, np.uint32)
    st, b, sizes, filled = oracle_mod.pocket_difference(g, st1, st2, bits, fill_volume=0.0)
    assert sizes.tolist() == [275.0] and filled.tolist() == [0]
    assert (st == 4).sum() == 275 and set(np.unique(st).tolist()) == {-1, 4}
    node_bits = np.unpackbits(b.view(np.uint8), bitorder="little")[:30 ** 3].reshape(30, 30, 30)
    assert 0 < node_bits[4:11, 5:12, 5:12].sum() == node_bits.sum() < 343
    assert node_bits[15:17, 15:17, 15:17].sum() == 0
    st_f, b_f, sizes_f, filled_f = oracle_mod.pocket_difference(g, st1, st2, bits, fill_volume=300.0)
    assert filled_f.tolist() == [1] and int(np.unpackbits(b_f.view(np.uint8)).sum()) == 0


def test_oracle_mesh_projection_known(oracle_mod):
    """MeshSurface::point2triangle on the unit right triangle: a point above the interior drops
    to its foot with the plane normal; a point beyond the corner B goes to B through the first
    edge (AB) and gets the reference's edge "normal" A + B t normalised, here (1, 0, 0)."""
    tri = [0, 0, 0, 1, 0, 0, 0, 1, 0]
    ins, proj, dist, nrm = oracle_mod.mesh_project([0.2, 0.2, 1.0], tri)
    assert ins and proj.tolist() == [0.2, 0.2, 0.0] and dist == 1.0 and nrm.tolist() == [0.0, 0.0, 1.0]
    ins, proj, dist, nrm = oracle_mod.mesh_project([2.0, -1.0, 0.5], tri)
    assert not ins and proj.tolist() == [1.0, 0.0, 0.0] and dist == 1.5 and nrm.tolist() == [1.0, 0.0, 0.0]
