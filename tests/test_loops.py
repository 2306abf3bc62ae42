"""While-loops over raster tests (the reference's symbolic loops,
python/map.py:234-330; runtime/Runtime.cpp:156-311) on scalar (D0) rasters,
which evaluate on the host: the loop forms, the caller's variables after the
loop, the test forms (`not`, `and`, `or`, Python values mixed in), nesting,
`else`, and the errors. Each loop is compared with the same loop over Python
numbers. Loops over 2-D rasters run on the GPU (test_gpu_loops.py)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture()
def L(M):
    return M


def test_scalar_loop_in_a_function(L):
    x = L.zeros(dt=L.S32)
    k = 0
    while x < 10:
        x = x + 3
        k += 1
    assert L.value(x) == 12 and k == 4


def test_not_test_and_loop_carried_python_values(L):
    y = L.zeros(dt=L.S32)
    seen = []
    while not (y >= 7):
        y = y + 1
        seen.append(1)
    assert L.value(y) == 7 and len(seen) == 7


@pytest.mark.parametrize("limit", [3, 100])
def test_and_with_a_python_value_first_and_last(L, limit):
    a = L.zeros(dt=L.F64)
    i = 0
    while i < limit and a < 5:
        a = a + 1.25
        i += 1
    ea, ei = 0.0, 0
    while ei < limit and ea < 5:
        ea, ei = ea + 1.25, ei + 1
    assert (L.value(a), i) == (ea, ei)
    b = L.zeros(dt=L.F64)
    j = 0
    while b < 5 and j < limit:
        b = b + 1.25
        j += 1
    assert (L.value(b), j) == (ea, ei)


def test_or_and_mixed_polarity(L):
    a = L.zeros(dt=L.S32)
    b = L.full(10, dt=L.S32)
    n = 0
    while a < 3 or not (b < 6):
        a = a + 1
        b = b - 1
        n += 1
    ea, eb, en = 0, 10, 0
    while ea < 3 or not (eb < 6):
        ea, eb, en = ea + 1, eb - 1, en + 1
    assert (L.value(a), L.value(b), n) == (ea, eb, en)
    c = L.zeros(dt=L.S32)
    while c < 4 and not (c > 2):
        c = c + 1
    assert L.value(c) == 3


def test_nested_loops_and_names_first_bound_in_the_body(L):
    a = L.zeros(dt=L.F64)
    i = 0
    while a < 5 and i < 100:
        b = a + 0.5
        j = L.zeros(dt=L.S32)
        while j < 3:
            j = j + 1
            b = b + 0.25
        a = b
        i += 1
    assert (L.value(a), i, L.value(j)) == (5.0, 4, 3)


def test_zero_iterations_and_else_clause(L):
    z = L.zeros(dt=L.S32)
    ran = []
    while z < 0:
        z = z + 1
    else:
        ran.append(L.value(z))
    assert ran == [0]


def test_invariant_and_in_place_update(L):
    step = L.full(2, dt=L.S32) * 1          # read, never assigned: kept resident once
    x = L.zeros(dt=L.S32)
    while x < 9:
        x = x + step
    assert L.value(x) == 10
    assert L.value(step) == 2


def test_loop_keeps_the_node_count_bounded(L):
    x = L.zeros(dt=L.S32)
    while x < 200:
        x = x + 1
    L.collect_garbage()
    assert L.value(x) == 200
    assert L.node_count() < 50


def test_truth_outside_a_loop(L):
    t = L.zeros(dt=L.S32) < 1
    assert bool(t) is True
    if L.zeros(dt=L.S32) > 0:
        raise AssertionError("a false scalar test was taken")


def test_errors(L):
    d2 = L.zeros([8, 8], dt=L.S32, bs=[8, 8])
    with pytest.raises(L.MapError, match="2-D raster"):
        bool(d2 < 1)
    x = L.zeros(dt=L.S32)
    with pytest.raises(L.MapError, match="break"):
        while x < 5:
            x = x + 1
            if x > 2:
                break


def test_materialize_scalars(L):
    a, b = L.materialize(L.zeros(dt=L.S32) + 4, L.ones(dt=L.F32) * 2.5)
    assert L.value(a) == 4 and L.value(b) == 2.5


def test_module_level_loop_and_source_less_fallback(tmp_path):
    """A loop at module level of a script writes the module's variables; a loop
    compiled from a string (no source file) runs in Python, test by test."""
    script = tmp_path / "loop_script.py"
    script.write_text(
        "from map import *\n"
        "x = zeros(dt=S32)\n"
        "k = 0\n"
        "while x < 10:\n"
        "    x = x + 3\n"
        "    k += 1\n"
        "ns = {}\n"
        "exec(compile('from map import *\\ny = zeros(dt=S32)\\nwhile y < 5:\\n    y = y + 2\\n', '<string>', 'exec'), ns)\n"
        "print(value(x), k, value(ns['y']))\n")
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "map_b200"))
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["12", "4", "6"]


_G = None


def test_global_and_nonlocal_names_assigned_in_the_loop(L):
    global _G
    _G = L.zeros(dt=L.S32)

    def bump():
        global _G
        n = 0
        while _G < 5:
            _G = _G + 1
            n += 1
        return n

    assert bump() == 5 and L.value(_G) == 5

    def outer():
        c = L.zeros(dt=L.S32)

        def inner():
            nonlocal c
            while c < 3:
                c = c + 1

        inner()
        return L.value(c)

    assert outer() == 3


def test_loop_in_a_method_and_tuple_assignment(L):
    class Acc:
        def run(self, k):
            a, b = L.zeros(dt=L.S32), L.ones(dt=L.S32)
            while b < k:
                a, b = b, a + b          # Fibonacci
            return L.value(a), L.value(b)

    assert Acc().run(50) == (34, 55)


def test_materialize_constants_pass_through_and_device_errors_are_reported(L):
    """A constant raster comes back as it is (nothing to evaluate); a computed
    2-D raster needs the device: without one the error is reported and the
    library stays usable."""
    a = L.zeros([8, 8], dt=L.S32, bs=[8, 8])
    (b,) = L.materialize(a)
    assert b._node.value == a._node.value
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(L.MapError):
            L.materialize(a + 1)
    assert L.value(L.materialize(L.zeros(dt=L.S32) + 2)[0]) == 2
