"""Fusion compiler and code generation on CPU: the reference scripts partition
into the groups the reference's fusion rules give, the plain-mode schedule
respects block dependencies, and every generated kernel compiles for sm_100a
with NVRTC (no device needed)."""
import numpy as np
import pytest

from map_b200 import workloads as W


def groups(M, *rs):
    return [l for l in M.describe_groups(*rs).splitlines() if l.strip()]


def nodes_of(line):
    return line.split("nodes=[")[1].split("]")[0]


def test_hillshade_is_one_focal_group(M):
    dem = M.from_numpy(np.zeros((64, 96), np.float32), bs=[32, 32])
    hs = W.hillshade(dem)
    g = groups(M, hs)
    assert len(g) == 1 and g[0].startswith("Focal")
    assert nodes_of(g[0]).count("Convolution") == 2          # both Sobel kernels share one staged tile
    assert M.compile_only(hs) == 1


def test_life_is_one_focal_group_per_generation(M):
    st = M.from_numpy(np.zeros((64, 64), np.uint8), bs=[32, 32])
    out = W.life(st, 5)
    g = groups(M, out)
    assert len(g) == 5 and all(x.startswith("Focal") for x in g)
    # every generation has the same structure, hence the same kernel source
    src = M.generated_source(out).split("//----")
    assert len(set(s.strip() for s in src if s.strip())) == 1


def test_stats_groups(M):
    dem = M.from_numpy(np.ones((64, 64), np.float32), bs=[32, 32])
    s = W.stats(dem)
    g = groups(M, *s.values())
    zonal = [x for x in g if x.startswith("Zonal")]
    host = [x for x in g if x.startswith("Host")]
    # all reductions of the raster itself flat-fuse into one pass; the deviation
    # pass (needs the mean) is a second zonal pass
    assert len(zonal) == 2
    assert nodes_of(zonal[0]).count("ZonalReduc") == 7
    assert nodes_of(zonal[1]).count("ZonalReduc") == 2
    assert len(host) >= 8


def test_wsum_is_one_local_group(M):
    ls = [M.from_numpy(np.zeros((16, 16), np.float32)) for _ in range(6)]
    out = W.wsum(ls, [0.1, 0.2, 0.3, 0.15, 0.15, 0.1])
    g = groups(M, out)
    assert len(g) == 1 and g[0].startswith("Local")


def test_focal_of_local_is_not_fused(M):
    d = M.from_numpy(np.zeros((16, 16), np.float32))
    out = M.convolve(d * 2.0, [[1, 1, 1]] * 3) + 1.0
    g = groups(M, out)
    assert [x.split()[0] for x in g] == ["Local", "Focal"]   # PIPE(LOCAL, FOCAL) is not allowed


def test_plain_schedule_respects_dependencies(M):
    st = M.from_numpy(np.zeros((96, 64), np.uint8), bs=[32, 32])
    out = W.life(st, 3)
    jobs = M.plain_schedule(out)
    nb = (2, 3)
    assert len(jobs) == 3 * nb[0] * nb[1]
    done = set()
    for g, bx, by, kind in jobs:
        if g > 0:
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    x, y = bx + dx, by + dy
                    if 0 <= x < nb[0] and 0 <= y < nb[1]:
                        assert (g - 1, x, y) in done, (g, bx, by)
        done.add((g, bx, by))
    # the schedule interleaves generations (it is not group-major)
    first_g1 = next(i for i, j in enumerate(jobs) if j[0] == 1)
    last_g0 = max(i for i, j in enumerate(jobs) if j[0] == 0)
    assert first_g1 < last_g0


@pytest.mark.parametrize("dt", ["U8", "S16", "S32", "U32", "F32", "F64", "S64"])
def test_generated_elementwise_kernels_compile(M, dt):
    npdt = {"U8": np.uint8, "S16": np.int16, "S32": np.int32, "U32": np.uint32, "F32": np.float32,
            "F64": np.float64, "S64": np.int64}[dt]
    a = M.from_numpy(np.ones((16, 16), npdt))
    b = M.from_numpy(np.ones((16, 16), npdt))
    exprs = [a + b, a - b, a * b, a / (b + 1), M.max(a, b), M.min(a, 3), a < b, M.con(a > b, a, b),
             M.astype(a, M.F32), (a == 1) * 2]
    if dt in ("F32", "F64"):
        exprs += [M.sin(a), M.atan2(a, b), M.sqrt(M.abs(a)), a ** b, M.exp(a) + M.log(b + 2)]
    else:
        exprs += [a % (b + 1)]
    if dt in ("U8", "U32"):
        one = M.full(1, [], a.datatype())
        exprs += [a & b, a | b, a ^ b, a << one, ~a]
    assert M.compile_only(*exprs) >= 1


def test_focal_variants_compile(M):
    d = M.from_numpy(np.zeros((40, 40), np.float32))
    u = M.from_numpy(np.zeros((40, 40), np.uint8))
    outs = [M.convolve(d, [[1.0 / 16, 1.0 / 8, 1.0 / 16], [1.0 / 8, 1.0 / 4, 1.0 / 8], [1.0 / 16, 1.0 / 8, 1.0 / 16]]),
            M.convolve(d, [[1] * 5] * 5), M.fmin(d, [[1] * 3] * 3), M.fmax(u, [[1] * 5] * 3), d([1, -1]) - d([0, 2]),
            M.flow_direction(d), M.convolve(u, [[1, 1, 1], [1, 0, 1], [1, 1, 1]])]
    assert M.compile_only(*outs) >= 1


def test_every_skeleton_compiles(M):
    """Zonal, radiating, spreading, rand and host-scalar programs generate
    kernels that NVRTC compiles for sm_100a."""
    dem = M.from_numpy(np.ones((40, 50), np.float32), bs=[32, 32])
    s = W.stats(dem)
    assert M.compile_only(*s.values()) == 2
    assert M.compile_only(W.life_initial([50, 40], [32, 32])) == 1
    v = W.viewshed(dem, [10, 20], 5.0)
    soft = M.convolve(v, [[1.0 / 16, 1.0 / 8, 1.0 / 16], [1.0 / 8, 1.0 / 4, 1.0 / 8], [1.0 / 16, 1.0 / 8, 1.0 / 16]])
    out = M.con(soft < 0.1, dem, M.zeros_like(dem))
    assert M.compile_only(out) >= 2
    d = M.flow_direction(dem)
    assert M.compile_only(M.flow_accumulation(M.ones_like(dem, M.S32), d)) == 2
    i64 = M.from_numpy(np.ones((8, 8), np.int64))
    assert M.compile_only(M.zsum(i64), M.zmax(M.from_numpy(np.ones((8, 8), np.uint8)))) == 2


def test_scalar_constants_become_literals(M):
    dem = M.from_numpy(np.zeros((16, 16), np.float32))
    src = M.generated_source(dem / 8 + 1.5)
    assert "a.s[" not in src and "/ ((s32)8)" in src


def test_sin_cos_pairs_share_sincosf(M):
    dem = M.from_numpy(np.zeros((16, 16), np.float32))
    x = M.atan(dem)
    src = M.generated_source(M.sin(x) * 2.0 + M.cos(x))
    import re
    assert "sincosf(" in src and not re.search(r"\bsinf\(", src) and not re.search(r"\bcosf\(", src)


def test_paired_cells_codegen(M):
    """Float focal groups get the two-rows-per-step form (focal_cell2) unless it is
    switched off, except the fast rewritten hillshade (one cell per step);
    integer focal groups on bytes (life) take the four-cell packed form. Every
    form compiles."""
    from map_b200 import workloads as W
    dem = M.from_numpy(np.zeros((64, 64), np.float32), bs=[32, 32])
    try:
        assert "focal_cell2" not in M.generated_source(W.hillshade(dem))     # fast form
        M.set_algebraic_rewrite(2)
        hs = W.hillshade(dem)
        assert "focal_cell2" in M.generated_source(hs)
        assert M.compile_only(hs) == 1
        M.set_paired_cells(False)
        assert not M.get_paired_cells()
        hs = W.hillshade(dem)
        assert "focal_cell2" not in M.generated_source(hs)
        assert M.compile_only(hs) == 1
    finally:
        M.set_paired_cells(True)
        M.set_algebraic_rewrite(1)
    grid = M.from_numpy(np.zeros((64, 64), np.uint8), bs=[32, 32])
    src = M.generated_source(W.life(grid, 1))
    assert "focal_cell2" not in src and "focal_cell4" in src


def test_scan_kernel_forms_codegen(M):
    """Radial groups carry the cluster form (KNAME_cl) beside the one-CTA forms;
    flow accumulation of 32-bit integers uses the packed (sum, pending) word,
    floats the separate in-degree array; every form compiles for sm_100a."""
    import re
    from map_b200 import workloads as W
    dem = M.from_numpy(np.zeros((64, 64), np.float32), bs=[32, 32])
    obs = [10, 20]
    r = M.rmax((dem - 10.0) / W.distance(dem, obs), obs)
    src = M.generated_source(r)
    assert re.search(r"map_radial_[0-9a-f]+_cl\(", src) and "barrier.cluster.arrive" in src
    assert M.compile_only(r) == 1
    d8 = M.flow_direction(dem)
    for dt, packed in ((M.S32, True), (M.U32, True), (M.F32, False)):
        acc = M.flow_accumulation(M.ones_like(dem, dt), d8)
        src = M.generated_source(acc)
        for k in ("_kahn(", "_kahn_many(", "_prep_many(", "_kahnp_many(", "_init("):
            assert re.search(r"map_spread_[0-9a-f]+" + re.escape(k), src), k
        assert ("spread_kahn_packed" in src) == packed
        assert ("spread_walk_packed" in src) == packed
        assert M.compile_only(acc) >= 1
