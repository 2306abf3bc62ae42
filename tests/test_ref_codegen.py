"""The oracle pinned on the reference's own code generator.

tests/golden/ref_kernel_facts.json holds facts of the OpenCL kernels that the
reference's runtime generates for the example programs (hill.py, life.py,
wsum.py, stats.py, view.py), and of the scalar values it launches them with,
produced by running
the reference's DAG, fusion compiler and kernel generators built from its own
sources (oracle/ref_codegen: build_ref_codegen.py, dump_kernels.py). These
tests check that the oracle's restatement (oracle/oracle.c) performs the same
operations in the same order with the same constants, and, where the
reference checkout is present, that the facts are what the reference
generates today."""
import json
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FACTS = os.path.join(ROOT, "tests", "golden", "ref_kernel_facts.json")


@pytest.fixture(scope="module")
def facts():
    with open(FACTS) as f:
        return json.load(f)


def core(kernels, n_loops):
    ks = [k for k in kernels if len(k["focal_loops"]) == n_loops]
    assert len(ks) >= 1
    return ks[0]


# hill_cell_f32 of oracle/oracle.c, statement by statement, in the facts'
# canonical names: t0 / t3 the two correlations, t5 the centre cell (unused),
# t6..t14 the scalar arguments (8, 1, cz, 0, 2 PI', 3 PI'/2, PI'/2, ar, sz)
HILL_ORACLE = [
    "t0f = 0", "t3f = 0", "t5f = LOAD_L_F32(IN)",
    "t6i = a0", "t7i = a1", "t8f = a2", "t9i = a3", "t10f = a4", "t11f = a5", "t12f = a6", "t13f = a7", "t14f = a8",
    "t15f = t0f / t6i",            # gx = ch / 8
    "t16f = t3f / t6i",            # gy = cv / 8
    "t17f = t16f * t16f",          # gy * gy
    "t18f = t15f * t15f",          # gx * gx
    "t19f = t18f + t17f",          # gx * gx + gy * gy
    "t20f = sqrt(t19f)",
    "t21f = t7i * t20f",           # 1 * sqrt(...)
    "t22f = atan(t21f)",           # s
    "t23f = cos(t22f)",
    "t24f = t8f * t23f",           # cz * cos(s)
    "t25f = -t15f",
    "t26f = atan2(t16f,t25f)",     # atan2(gy, -gx)
    "t27u8 = t15f != t9i",
    "t28f = t27u8 * t26f",         # z1
    "t29u8 = t28f < t9i",
    "t30f = t29u8 * t10f",
    "t31f = t28f + t30f",          # z1 += (z1 < 0) * 2 PI'
    "t32u8 = t16f < t9i",
    "t33f = t32u8 * t11f",         # (gy < 0) * 3 PI'/2
    "t34u8 = t16f > t9i",
    "t35f = t34u8 * t12f",         # (gy > 0) * PI'/2
    "t36f = t35f + t33f",
    "t37u8 = t15f == t9i",
    "t38f = t37u8 * t36f",         # z0
    "t39f = t31f + t38f",          # aspect
    "t40f = t13f - t39f",          # ar - aspect
    "t41f = cos(t40f)",
    "t42f = sin(t22f)",
    "t43f = t14f * t42f",          # sz * sin(s)
    "t44f = t43f * t41f",
    "t45f = t24f + t44f",          # hs
]


def strip_ids(stmts):
    import re
    return [re.sub(r"\(IN_\d+\)", "(IN)", s) for s in stmts]


def test_hillshade_restatement_matches_reference_kernel(facts):
    k = core(facts["hill"], 2)
    assert strip_ids(k["statements"]) == HILL_ORACLE
    # correlation: acc += tap * mask, rows (i1) outer, columns (i0) inner, integer masks
    assert k["loop_nesting"] == ["i1", "i0"]
    assert k["focal_loops"] == ["t0f += t1f[tap(i0,i1)] * t2i[i1][i0]", "t3f += t1f[tap(i0,i1)] * t4i[i1][i0]"]
    assert k["masks"]["t2i"] == [[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]]
    assert k["masks"]["t4i"] == [[-1, -2, -1], [0, 0, 0], [1, 2, 1]]


def test_hillshade_constants_are_the_oracles(facts):
    """The script's constants reach the reference kernel as exact float32 kernel
    arguments, equal to oracle.c's hill_const (Python double arithmetic, then
    float32)."""
    k = core(facts["hill"], 2)
    args = k["scalar_args"]
    assert [a["type"] for a in args] == ["int", "int", "float", "int", "float", "float", "float", "float", "float"]
    assert [args[i]["value"] for i in (0, 1, 3)] == [8, 1, 0]
    PI = 3.141593
    zr = (90 - 45.0) / 180 * PI
    ar = (360 - 315.0 + 90) / 180 * PI
    want = [math.cos(zr), PI * 2, PI * 2 - PI / 2, PI / 2, ar, math.sin(zr)]
    got = [args[i]["bits"] for i in (2, 4, 5, 6, 7, 8)]
    assert got == ["%08x" % np.float32(v).view(np.uint32) for v in want]


def test_life_restatement_matches_reference_kernel(facts):
    gens = [k for k in facts["life"] if len(k["focal_loops"]) == 1]
    assert len(gens) == 2       # two generations, one focal kernel each
    for k in gens:
        assert k["masks"]["t2i"] == [[1, 1, 1], [1, 0, 1], [1, 1, 1]]
        assert k["focal_loops"] == ["t0i += t1u8[tap(i0,i1)] * t2i[i1][i0]"]   # U8 taps, S32 accumulator
        assert k["loop_nesting"] == ["i1", "i0"]
        assert [a["value"] for a in k["scalar_args"]] == [2, 3]
        st = strip_ids(k["statements"])
        # (nbh == 3) + (nbh == 2) * state, all U8 (oracle.c orc_life)
        assert st[-4:] in (["t6u8 = t0i == t4i", "t7u8 = t6u8 * t3u8", "t8u8 = t0i == t5i", "t9u8 = t8u8 + t7u8"],
                           ["t6u8 = t0i == t3i", "t7u8 = t6u8 * t5u8", "t8u8 = t0i == t4i", "t9u8 = t8u8 + t7u8"])


def test_rand_key_and_counter_match_the_oracle(facts):
    """rand(seed, ...) > 128: Philox2x32 counter {seed}, key BS1*BC1 + BS0*BC0 +
    bc1*BS0 + bc0 (oracle.c orc_rand_u8), U8 draw = low byte of the counter."""
    k = [k for k in facts["life"] if k["rng"]][0]
    assert k["rng"] == ["philox2x32_ctr_t ctr = {{t1u8}};",
                        "philox2x32_key_t key = {{BS1*BC1+BS0*BC0+(bc1)*BS0+bc0}};",
                        "ctr = philox2x32(ctr,key);"]
    assert any(s.startswith("t2u8 = *(uchar*)& ctr") for s in k["statements"])
    assert [a["value"] for a in k["scalar_args"]] == [128]


def test_wsum_left_to_right(facts):
    k = facts["wsum"][0]
    st = strip_ids(k["statements"])
    # 0 + 0.1*r1 + r2*0.2 + 0.3*r3 + r4*0.4 + 0, left to right (oracle.c orc_wsum_f32)
    assert st[9:] == ["t9f = t4f * t0f", "t10f = t5i + t9f", "t11f = t1f * t6f", "t12f = t10f + t11f",
                      "t13f = t7f * t2f", "t14f = t12f + t13f", "t15f = t3f * t8f", "t16f = t14f + t15f",
                      "t17f = t16f + t5i"]
    vals = [a["value"] for a in k["scalar_args"]]
    assert vals == [np.float32(0.1), 0, np.float32(0.2), np.float32(0.3), np.float32(0.4)]


def test_facts_are_what_the_reference_generates():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref_codegen"))
    import build_ref_codegen as B
    import dump_kernels as D
    if not os.path.isfile(os.path.join(B.REF, "Makefile")):
        pytest.skip("reference checkout not available")
    exe = B.build()
    with open(FACTS) as f:
        committed = json.load(f)
    assert json.loads(json.dumps(D.facts(exe), sort_keys=True)) == committed


def _ref_exe():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref_codegen"))
    import build_ref_codegen as B
    if not os.path.isfile(os.path.join(B.REF, "Makefile")):
        pytest.skip("reference checkout not available")
    return B.build()


def _pattern(w, h, dtype):
    y, x = np.mgrid[0:h, 0:w]
    v = ((x * 7 + y * 13) % 251).astype(np.float64) + 0.25 * (x % 4)
    return v.astype(dtype)


@pytest.mark.parametrize("w,h,bs,dt", [(300, 200, 128, 1), (256, 256, 256, 4), (257, 130, 64, 10)])
def test_bin_files_written_by_the_reference_read_here(M, tmp_path, w, h, bs, dt):
    """The reference's own .bin writer (file/binary.cpp File<binary>, block by
    block) produces files this engine reads cell for cell."""
    import subprocess
    exe = _ref_exe()
    path = str(tmp_path / "ref.bin")
    subprocess.run([exe, "binwrite", path, str(w), str(h), str(bs), str(dt)], check=True, timeout=60,
                   stdout=subprocess.DEVNULL)
    np_dt = {1: np.float32, 4: np.uint8, 10: np.int32}[dt]
    got = M.bin_read_numpy(path)
    assert got.dtype == np_dt and got.shape == (h, w)
    assert np.array_equal(got, _pattern(w, h, np_dt))


@pytest.mark.parametrize("w,h,bs,dtype", [(300, 200, (128, 128), np.float32), (257, 130, (64, 32), np.uint8),
                                          (100, 100, (100, 100), np.int32)])
def test_bin_files_written_here_read_by_the_reference(M, tmp_path, w, h, bs, dtype):
    """Files this engine writes are read back by the reference's own reader
    (File<binary>::readBlock) with the same header and cells."""
    import subprocess
    exe = _ref_exe()
    a = (np.random.default_rng(3).random((h, w)) * 200).astype(dtype)
    path, dense = str(tmp_path / "ours.bin"), str(tmp_path / "dense")
    M.bin_write_numpy(path, a, bs=bs)
    subprocess.run([exe, "binread", path, dense], check=True, timeout=60, stdout=subprocess.DEVNULL)
    raw = open(dense, "rb").read()
    head, body = raw.split(b"\n", 1)
    dt, W, H, mo, b0, b1 = map(int, head.split())
    assert (W, H, b0, b1) == (w, h) + tuple(bs)
    assert mo == M.ROW + M.BLK and dt == M._dt_of_np[np.dtype(dtype).name]
    assert np.array_equal(np.frombuffer(body, dtype=dtype).reshape(h, w), a)


def test_stats_reductions_as_the_reference_generates_them(facts, M):
    """stats.py (python/stats.py:12-35): the reference's two zonal kernels
    reduce with these neutral values and operators (util/ReductionType.cpp),
    compute 1.0 / dem, dem ** 2 and dem ** 3 as pow with an integer exponent,
    and in the second pass (dem - mean) ** 2 and (dev - minv) / rang; the
    engine's kernels for the same script start from the same neutral values
    and compute the same operations."""
    first, second = facts["stats"]
    assert first["statements"][4:] == ["t4f = t1f / t0f", "t5f = pow(t0f,t2i)", "t6f = pow(t0f,t3i)"]
    assert [(a["type"], a["value"]) for a in first["scalar_args"]] == [("float", 1.0), ("int", 2), ("int", 3)]
    assert first["zonal"] == [{"atomic": "MAX", "tree": "max", "neutral": "-INFINITY"},
                              {"atomic": "MIN", "tree": "min", "neutral": "INFINITY"},
                              {"atomic": "SUM", "tree": "+", "neutral": "0"},
                              {"atomic": "PROD", "tree": "*", "neutral": "1"}] + \
        [{"atomic": "SUM", "tree": "+", "neutral": "0"}] * 3
    assert second["statements"][5:] == ["t5f = t0f - t3f", "t6f = pow(t5f,t4i)", "t7f = t6f - t1f", "t8f = t7f / t2f"]
    assert [z["atomic"] for z in second["zonal"]] == ["SUM", "SUM"]
    import re
    src = M.generated_source(*W_stats(M).values())
    for red, neutral in ((6, "__int_as_float(0xff800000)"), (7, "__int_as_float(0x7f800000)"), (1, "0x0p+0f"),
                         (2, "0x1p+0f")):
        acc = re.search(r"(acc\d+) = RedOp<%d, float>" % red, src).group(1)
        assert re.search(r"float %s = %s;" % (acc, re.escape(neutral)), src), (red, neutral)
    assert re.search(r"= \(float\)\(\(\(float\)0x1p\+0f\) / i0\);", src)           # 1.0 / dem in float32
    assert len(re.findall(r"powf\(\(float\)\(\w+\), \(float\)\(\(\(s32\)2\)\)\)", src)) == 2   # dem ** 2, dev
    assert len(re.findall(r"powf\(\(float\)\(\w+\), \(float\)\(\(\(s32\)3\)\)\)", src)) == 1


def W_stats(M):
    import numpy as np
    from map_b200 import workloads as W
    return W.stats(M.from_numpy(np.ones((512, 512), np.float32), bs=[256, 256]))


def test_viewshed_chain_as_the_reference_generates_it(facts):
    """view.py (python/view.py:17-43): the reference's radial kernel computes
    the normalised DEM, the observer distance with S64 integer differences and
    squares (x*x + y*y), converted to F32 by the + 0.0, its square root, the
    slope, the radial max guarded by isfinite, and the view; the restatement
    the tests use (tests/test_gpu_scan.py slope_from_observer, oracle.c
    orc_radial_f32) follows those steps, checked here by evaluating the
    reference's statements literally in NumPy against it."""
    import importlib.util
    import numpy as np
    radial = [k for k in facts["view"] if k["guards"]][0]
    assert radial["guards"] == ["isfinite(t19f)"]
    st = radial["statements"]
    assert st[7:] == ["t7f = t0f - t1f", "t8f = t7f / t2f", "t9f = t8f - t3f", "t10l = BC0*BS0+bc0", "t11l = t4i - t10l",
                      "t12l = BC1*BS1+bc1", "t13l = t5i - t12l", "t14l = t13l * t13l", "t15l = t11l * t11l",
                      "t16l = t15l + t14l", "t17f = t16l + t6f", "t18f = sqrt(t17f)", "t19f = t9f / t18f",
                      "t20f = LIT_F32(t21f[gc+1],t21f[gc])", "t20f = max(t20f, t19f)", "t22f = t20f * t18f",
                      "t23f = t22f + t3f", "t24f = t23f - t8f"]
    args = radial["scalar_args"]
    assert [a["type"] for a in args] == ["float", "float", "float", "int", "int", "float"]
    assert args[2]["bits"] == "41200000" and [args[3]["value"], args[4]["value"]] == [100, 150]
    assert args[5]["bits"] == "00000000"
    # the reference's statements, literally, on a small normalised raster
    rng = np.random.default_rng(3)
    h, w, ox, oy, hh = 37, 53, 11, 29, np.float32(10.0)
    norm = rng.random((h, w)).astype(np.float32)
    t10 = np.arange(w, dtype=np.int64)[None, :]
    t12 = np.arange(h, dtype=np.int64)[:, None]
    t11, t13 = np.int64(ox) - t10, np.int64(oy) - t12
    t16 = t11 * t11 + t13 * t13
    t17 = (t16.astype(np.float32) + np.float32(0.0)).astype(np.float32)
    t18 = np.sqrt(t17)
    with np.errstate(divide="ignore", invalid="ignore"):
        t19 = ((norm - hh) / t18).astype(np.float32)
    spec = importlib.util.spec_from_file_location("gpu_scan", os.path.join(ROOT, "tests", "test_gpu_scan.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    slope, dist = mod.slope_from_observer(norm, [ox, oy], 10.0)
    assert np.array_equal(dist.view(np.uint32), t18.view(np.uint32))
    assert np.array_equal(slope.view(np.uint32), t19.view(np.uint32))
    focal = [k for k in facts["view"] if k["masks"]][0]
    assert list(focal["masks"].values()) == [[[0.0625, 0.125, 0.0625], [0.125, 0.25, 0.125], [0.0625, 0.125, 0.0625]]]
    assert focal["statements"][-2:] == ["t7u8 = t0f < t5f", "t8f = (t7u8) ? t3f : t6f"]    # con(soft < 0.1, dem, 0)
    assert focal["scalar_args"] == [{"type": "float", "value": np.float32(0.1).item(), "bits": "3dcccccd"}]


def test_focal_percent_as_the_reference_generates_it(facts):
    """FocalPercent (front/Raster.cpp:438-447, runtime/skeleton/FocalSkeleton.cpp:
    375-403) as the reference generates it cannot run: its halo sizes are
    empty (`int H0 = ;`), its window loops start at the centre (0 .. 2h), its
    divisor lacks parentheses ((H0*2+1)*H1*2+1 instead of the window size), it
    compares against the centre value before loading it (the load follows the
    core), and its Predictor asserts on the node. The oracle keeps what the
    kernel states -- `==` for percentage, `>` for percentile, a count in the
    argument's type from 0, divided after the loop -- over the window centred
    on the cell, by the window size, against the cell's own value."""
    import numpy as np
    from oracle import oracle as O
    (k,) = facts["percent"]
    assert k["halo"] == ["int H0 = ;", "int H1 = ;"]
    assert k["loop_headers"] == ["for (int i1=0; i1<3; i1++)", "for (int i0=0; i0<3; i0++)"] * 2
    assert k["focal_loops"] == ["t0f += (t1f == t2f[tap(i0,i1)])", "t3f += (t1f > t2f[tap(i0,i1)])"]
    assert k["scalings"] == ["t0f /= (H0*2+1)*H1*2+1", "t3f /= (H0*2+1)*H1*2+1"]
    assert k["statements"][:3] == ["t0f = 0", "t3f = 0", "t1f = LOAD_L_F32(IN_6)"]
    a = np.random.default_rng(1).integers(0, 3, (20, 30)).astype(np.float32)
    p = np.pad(a, 1)
    win = np.stack([p[i:i + 20, j:j + 30] for i in range(3) for j in range(3)])
    for typ, cmp in ((1, np.equal), (2, np.greater)):
        want = (cmp(a[None], win).astype(np.float32).sum(axis=0) / np.float32(9)).astype(np.float32)
        got = O.focal_percent(a, 1, 1, typ, (64, 64), border=2)
        inner = (slice(1, -1), slice(1, -1))
        assert np.array_equal(got[inner], want[inner])
