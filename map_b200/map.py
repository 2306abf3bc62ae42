##
# Python 3 interface of the B200 map-algebra engine over its C ABI (ctypes).
#
# Same module surface as the reference's Python bindings (python/map.py): the
# enum tables, Variant / Array / Node / Raster, operator overloading, the
# module functions (read, write, eval, value, convolve, zsum, rmax, con, ...)
# and the compound helpers, so scripts written for it (`from map import *`)
# run unchanged under Python 3 when this directory is on sys.path.
#
# Differences from the reference module:
#  * Python 3: `/` maps to __truediv__, `__bool__` replaces `__nonzero__`;
#  * errors raise MapError with the library's message instead of asserting;
#  * while-loops over raster tests (python/map.py:234-330) are run by this
#    module, one evaluation per iteration with loop-carried rasters kept
#    resident, where the reference only captures them (its runtime has no task
#    to execute them);
#  * extensions at the end: NumPy in/out, border and launch-mode switches,
#    device-resident inputs, flow direction / accumulation and viewshed helpers.
##

import builtins as _builtins
import ctypes as ct
import functools
import math
import operator
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.environ.get("MAP_B200_LIB", os.path.join(_HERE, "libmap_b200.so"))
if not os.path.exists(_LIBPATH):
    raise ImportError("map: native library %s is missing; build it with `python -m map_b200.build`" % _LIBPATH)
_lib = ct.CDLL(_LIBPATH)


class MapError(RuntimeError):
    pass


## Enumerates / Constants (python/map.py:35-90)

DataTypeId = ['NONE_DATATYPE', 'F32', 'F64', 'B8', 'U8', 'U16', 'U32', 'U64', 'S8', 'S16', 'S32', 'S64', 'N_DATATYPE']
DataTypeVal = list(range(len(DataTypeId)))

NumDimId = ['NONE_NUMDIM', 'TIME', 'D0', 'D1', 'D2', 'D3', 'N_NUMDIM']
NumDimVal = [0x00, 0x01, 0x02, 0x04, 0x06, 0x08, 0x0A]

MemOrderId = ['NONE_MEMORDER', 'BLK', 'ROW', 'COL', 'SFC', 'N_MEMORDER']
MemOrderVal = [0x00, 0x01, 0x02, 0x04, 0x06, 0x08]

DeviceTypeId = ['DEV_DEF', 'DEV_CPU', 'DEV_GPU', 'DEV_ACC', 'DEV_CUS', 'DEV_ALL']
DeviceTypeVal = [0x01, 0x02, 0x04, 0x08, 0x16, 0xFFFFFFFF]

UnaryTypeId = [
    'NONE_UNARY', 'POS', 'NEG', 'NOT', 'bNOT', 'MARK_UNARY',
    'SIN', 'COS', 'TAN', 'ASIN', 'ACOS', 'ATAN',
    'SINH', 'COSH', 'TANH', 'ASINH', 'ACOSH', 'ATANH',
    'EXP', 'EXP2', 'EXP10', 'LOG', 'LOG2', 'LOG10',
    'SQRT', 'CBRT', 'ABS',
    'CEIL', 'FLOOR', 'TRUNC', 'ROUND', 'N_UNARY'
]
UnaryTypeSym = [
    '', '__pos__', '__neg__', '__not__', '__invert__', '',
    'sin', 'cos', 'tan', 'asin', 'acos', 'atan',
    'sinh', 'cosh', 'tanh', 'asinh', 'acosh', 'atanh',
    'exp', 'exp2', 'exp10', 'log', 'log2', 'log10',
    'sqrt', 'cbrt', 'abs',
    'ceil', 'floor', 'trunc', 'round', ''
]
UnaryTypeVal = list(range(len(UnaryTypeId)))

BinaryTypeId = [
    'NONE_BINARY', 'ADD', 'SUB', 'MUL', 'DIV', 'MOD',
    'EQ', 'NE', 'LT', 'GT', 'LE', 'GE', 'AND', 'OR',
    'bAND', 'bOR', 'bXOR', 'SHL', 'SHR', 'MARK_BINARY',
    'MAX2', 'MIN2', 'ATAN2', 'POW', 'HYPOT', 'FMOD', 'N_BINARY'
]
BinaryTypeSym = [
    '', '__add__', '__sub__', '__mul__', '__truediv__', '__mod__',
    '__eq__', '__ne__', '__lt__', '__gt__', '__le__', '__ge__', '', '',
    '__and__', '__or__', '__xor__', '__lshift__', '__rshift__', '',
    'max', 'min', 'atan2', 'pow', 'hypot', 'fmod', ''
]
BinaryTypeVal = list(range(len(BinaryTypeId)))

ReductionTypeId = ['NONE_REDUCTION', 'SUM', 'PROD', 'rAND', 'rOR', 'MARK_REDUCTION', 'MAX', 'MIN', 'N_REDUCTION']
ReductionTypeVal = list(range(len(ReductionTypeId)))

EnumIds = [DataTypeId, NumDimId, MemOrderId, DeviceTypeId, UnaryTypeId, BinaryTypeId, ReductionTypeId]
EnumVals = [DataTypeVal, NumDimVal, MemOrderVal, DeviceTypeVal, UnaryTypeVal, BinaryTypeVal, ReductionTypeVal]

for _ids, _vals in zip(EnumIds, EnumVals):
    for _i, _v in zip(_ids, _vals):
        globals()[_i] = _v

# border rules and launch modes (extensions)
BORDER_BLOCK_MIRROR, BORDER_RASTER_MIRROR, BORDER_DEAD = 0, 1, 2
EXEC_FUSED, EXEC_PLAIN = 0, 1

## Wrapper classes


class Variant(ct.Structure):
    class Union(ct.Union):
        _fields_ = [
            ('b8', ct.c_bool), ('s8', ct.c_int8), ('s16', ct.c_int16), ('s32', ct.c_int32), ('s64', ct.c_int64),
            ('u8', ct.c_uint8), ('u16', ct.c_uint16), ('u32', ct.c_uint32), ('u64', ct.c_uint64),
            ('f16', ct.c_float), ('f32', ct.c_float), ('f64', ct.c_double)
        ]
    _fields_ = [('union', Union), ('dtype', ct.c_int)]

    _field_of = {F32: 'f32', F64: 'f64', B8: 'b8', U8: 'u8', U16: 'u16', U32: 'u32', U64: 'u64',
                 S8: 's8', S16: 's16', S32: 's32', S64: 's64'}

    def __init__(self, val=None, dtype=None):
        union = self.Union()
        if val is None:
            super().__init__(union, NONE_DATATYPE)
            return
        if dtype is not None:
            setattr(union, self._field_of[dtype], val)
            super().__init__(union, dtype)
            return
        if isinstance(val, float):
            union.f32, dtype = val, F32
        elif isinstance(val, bool):
            union.b8, dtype = val, B8
        elif isinstance(val, int):
            union.s32, dtype = val, S32
        elif isinstance(val, ct.c_uint8):
            union.u8, dtype = val.value, U8
        else:
            raise MapError("Variant: unsupported value %r" % (val,))
        super().__init__(union, dtype)

    def datatype(self):
        return self.dtype

    def value(self):
        f = self._field_of.get(self.dtype)
        if f is None:
            raise MapError("Variant has no value")
        return getattr(self.union, f)

    def convert(self, new_dt):
        v = self.value()
        if new_dt in (F32, F64):
            return Variant(float(v), new_dt)
        if new_dt == B8:
            return Variant(bool(v), B8)
        return Variant(int(v), new_dt)


class Array(ct.Structure):
    N = 2
    T = ct.c_int * N
    _fields_ = [('arr', T), ('n', ct.c_int)]

    def __init__(self, arg=()):
        if arg is None or (isinstance(arg, (list, tuple)) and len(arg) == 0):
            super().__init__(self.T(-1, -1), 0)
        elif isinstance(arg, (list, tuple)):
            if len(arg) != self.N:
                raise MapError("Array needs %d elements, got %d" % (self.N, len(arg)))
            super().__init__(self.T(*[int(a) for a in arg]), self.N)
        elif isinstance(arg, Array):
            super().__init__(arg.arr, arg.n)
        else:
            raise MapError("Array: unsupported argument %r" % (arg,))

    def isNone(self):
        return all(e == -1 for e in self.arr)

    def toList(self):
        return [x for x in self.arr if x != -1]


class Node(ct.c_void_p):  # distinct type so ctypes returns a handle, not an int
    pass


def _check(result, func, args):
    if _lib.ma_errorCode():
        raise MapError(_lib.ma_lastError().decode())
    return result


class Raster:
    def __init__(self, node=None):
        if isinstance(node, Node):
            if not node.value:
                raise MapError("null node")
            self._node = node
            _lib.ma_increaseRef(self)
        elif node is None:
            self._node = Node(None)
        else:
            raise MapError("Raster: expected a node handle")

    def __del__(self):
        try:
            if getattr(self, "_node", None) is not None and self._node.value:
                _lib.ma_decreaseRef(self)
        except Exception:
            pass

    @classmethod
    def from_param(cls, ins):  # lets ctypes take ._node from Rasters given as arguments
        return ins._node

    def __getitem__(self, key):
        if isinstance(key, (list, tuple)):
            return Raster(_lib.ma_access(self, Array(key)))
        elif isinstance(key, Raster):
            return Raster(_lib.ma_conditional(key, self, empty_like(self)))
        raise MapError("unsupported index")

    def __setitem__(self, key, other):
        other = _const_to_raster(other).astype(self.datatype())
        if isinstance(key, (list, tuple)):
            node = _lib.ma_lhsAccess(self, other, Array(key))
        elif isinstance(key, Raster):
            node = _lib.ma_conditional(key, other, self)
        else:
            raise MapError("unsupported index")
        _lib.ma_increaseRef(node)
        _lib.ma_decreaseRef(self)
        self._node = node

    def __call__(self, ngb):
        if isinstance(ngb, list):
            return Raster(_lib.ma_neighbor(self, Array(ngb)))
        elif isinstance(ngb, tuple):
            if len(ngb) != 2 or not isinstance(ngb[0], Raster):
                raise MapError("bounded neighbourhood needs two rasters")
            return Raster(_lib.ma_boundedNbh(self, ngb[0], ngb[1]))
        raise MapError("unsupported neighbour access")

    def __bool__(self):
        # Truth value of a scalar (D0) raster, evaluated. In the test of a
        # `while` statement whose source file is readable, the whole loop runs
        # here instead (_run_while: the reference's hook for symbolic loops,
        # python/map.py:234-330) and the value returned makes the test false.
        if _lib.ma_numdim(self) != D0:
            raise MapError("the truth value of a 2-D raster is ambiguous: reduce it to a scalar (D0) raster first, "
                           "e.g. with zmax or zor")
        replay = getattr(_loop_tls, "replay", None)
        if replay is not None:
            return replay.answer(self)
        if getattr(_loop_tls, "truth", 0) > 0:
            return _truth_of(self)
        frame = _sys._getframe(1)
        loop = _while_at(frame)
        if loop is None:
            return _truth_of(self)
        # A raster asked for later in the same evaluation of the test (a larger
        # instruction offset than the request that ran the loop) belongs to the
        # test the loop's answer ends: its own truth, no second loop.
        done = _loop_tls.__dict__.setdefault("done", {})
        key = (id(frame), frame.f_code.co_filename, loop.lineno)
        last = done.pop(key, None)
        if last is not None and frame.f_lasti > last:
            done[key] = last
            return _truth_of(self)
        r = _run_while(loop, frame)
        if len(done) > 64:
            done.clear()
        done[key] = frame.f_lasti
        return r

    __hash__ = object.__hash__

    ## Public methods

    def nodeid(self):
        return _lib.ma_nodeid(self)

    def streamdir(self):
        return _lib.ma_streamdir(self)

    def datatype(self):
        return _lib.ma_datatype(self)

    def numdim(self):
        return _lib.ma_numdim(self)

    def memorder(self):
        return _lib.ma_memorder(self)

    def datasize(self):
        return _lib.ma_datasize(self).toList()

    def blocksize(self):
        return _lib.ma_blocksize(self).toList()

    def numblock(self):
        return _lib.ma_numblock(self).toList()

    def __pow__(self, other):
        rhs = _const_to_raster(other)
        return Raster(_lib.ma_binary(self, rhs, POW))

    def __rpow__(self, other):
        lhs = _const_to_raster(other)
        return Raster(_lib.ma_binary(lhs, self, POW))

    def no(self):
        return Raster(_lib.ma_unary(self, NOT))

    def astype(self, dt):
        return astype(self, dt)

    # extensions
    def numpy(self):
        return to_numpy(self)


## Helper functions

def _const_to_raster(arg):
    if isinstance(arg, Raster):
        return arg
    elif isinstance(arg, (bool, int, float)):
        var = Variant(arg)
        return Raster(_lib.ma_constant(var, Array(), var.datatype(), ROW + BLK, Array()))
    raise MapError("cannot convert %r to a raster" % (arg,))


## Unary functions

def _def_unary_op(symbol, utype):
    def uop(self):
        return Raster(_lib.ma_unary(self, utype))
    setattr(Raster, symbol, uop)


def _def_unary_fun(symbol, utype):
    def ufun(raster):
        if isinstance(raster, Raster):
            return Raster(_lib.ma_unary(raster, utype))
        if symbol == 'exp10':
            return 10.0 ** raster
        if symbol == 'round':
            return _builtins.round(raster)
        if symbol == 'abs':
            return _builtins.abs(raster)
        return getattr(math, symbol)(raster)
    globals()[symbol] = ufun


for _sym, _ut in zip(UnaryTypeSym, UnaryTypeVal):
    if _sym and _ut < MARK_UNARY:
        _def_unary_op(_sym, _ut)
    elif _sym and _ut > MARK_UNARY:
        _def_unary_fun(_sym, _ut)

## Binary functions


def _def_binary_op(symbol, bitype):
    def biop(self, rhs):
        rhs = _const_to_raster(rhs)
        return Raster(_lib.ma_binary(self, rhs, bitype))
    setattr(Raster, symbol, biop)

    def rbiop(self, lhs):
        lhs = _const_to_raster(lhs)
        return Raster(_lib.ma_binary(lhs, self, bitype))
    rsymbol = symbol[:2] + 'r' + symbol[2:]
    setattr(Raster, rsymbol, rbiop)


def _def_binary_fun(symbol, bitype):
    def bifun(lhs, rhs):
        if not isinstance(lhs, Raster) and not isinstance(rhs, Raster):
            if symbol == 'max':
                return _builtins.max(lhs, rhs)
            if symbol == 'min':
                return _builtins.min(lhs, rhs)
            return getattr(math, symbol)(lhs, rhs)
        lhs = _const_to_raster(lhs)
        rhs = _const_to_raster(rhs)
        return Raster(_lib.ma_binary(lhs, rhs, bitype))
    globals()[symbol] = bifun


for _sym, _bt in zip(BinaryTypeSym, BinaryTypeVal):
    if _sym and _bt < MARK_BINARY:
        _def_binary_op(_sym, _bt)
    elif _sym and _bt > MARK_BINARY:
        _def_binary_fun(_sym, _bt)

# Python 2 spelling of the division operator, kept for callers that use it
Raster.__div__ = Raster.__truediv__
Raster.__rdiv__ = Raster.__rtruediv__

## While-loops over rasters (python/map.py:234-330, runtime/Runtime.cpp:156-311)
#
# When Python asks for the truth value of a raster in a `while` test, the
# reference re-reads the loop's source from the caller's file (inspect + ast),
# runs the body twice symbolically to find the loop-carried values and builds
# Loop nodes, which its runtime has no task to execute. Here the same hook runs
# the loop: the test and the body, compiled from the caller's file, are
# evaluated in the caller's namespace, one evaluation per iteration. Every
# raster the body assigns (loop-carried) and every raster the loop reads but
# does not assign (invariant) is kept resident through materialize(), so an
# iteration evaluates only its own body, the test's reduction fused with it.
# Afterwards the caller's variables hold the last iteration's values and the
# hook returns the truth value that makes the caller's test false (found by
# replaying the test), so Python leaves the loop (and runs its `else` clause).
# `break`, `continue`, `return` and `yield` directly in such a body are not
# supported; the test is evaluated more than once and should have no side
# effects. Without a readable source (interactive input, exec of a string) a
# raster test is just evaluated each time Python asks: the loop runs in
# Python, correct but recomputing the loop's history at every test.

import ast as _ast
import linecache as _linecache
import sys as _sys
import threading as _threading

_loop_tls = _threading.local()
_tree_cache = {}


def _truth_of(r):
    _lib.ma_eval(ct.cast((Node * 1)(r._node), ct.POINTER(Node)), 1)
    return bool(_lib.ma_value(r).value())


def _file_tree(filename, module_globals):
    lines = _linecache.getlines(filename, module_globals)
    if not lines:
        return None
    text = "".join(lines)
    key = (filename, hash(text))
    tree = _tree_cache.get(key)
    if tree is None:
        try:
            tree = _ast.parse(text, filename)
        except SyntaxError:
            return None
        if len(_tree_cache) > 32:
            _tree_cache.clear()
        _tree_cache[key] = tree
    return tree


def _while_at(frame):
    """The innermost `while` statement of the frame's file whose test spans the
    frame's current line, or None."""
    filename = frame.f_code.co_filename
    if filename.startswith("<"):
        return None
    tree = _file_tree(filename, frame.f_globals)
    if tree is None:
        return None
    line = frame.f_lineno
    spans = _while_spans.get(id(tree))
    if spans is None or spans[0] is not tree:
        tests = [n for n in _ast.walk(tree) if isinstance(n, _ast.While)]
        spans = (tree, {})
        for n in tests:
            for l in range(n.test.lineno, n.test.end_lineno + 1):
                b = spans[1].get(l)
                if b is None or n.lineno > b.lineno:       # the innermost statement
                    spans[1][l] = n
        if len(_while_spans) > 32:
            _while_spans.clear()
        _while_spans[id(tree)] = spans
    return spans[1].get(line)


_while_spans = {}   # id(tree) -> (tree, {line: innermost while statement whose test spans it})


def _target_names(t, out):
    if isinstance(t, _ast.Name):
        out.add(t.id)
    elif isinstance(t, (_ast.Tuple, _ast.List)):
        for e in t.elts:
            _target_names(e, out)
    elif isinstance(t, _ast.Starred):
        _target_names(t.value, out)
    elif isinstance(t, (_ast.Subscript, _ast.Attribute)):   # x[m] = v updates the raster x in place
        _target_names(t.value, out)


def _loop_names(loop):
    """(names the body assigns, names the test or body reads)."""
    assigned, read = set(), set()
    for stmt in loop.body:
        for n in _ast.walk(stmt):
            if isinstance(n, (_ast.Assign,)):
                for t in n.targets:
                    _target_names(t, assigned)
            elif isinstance(n, (_ast.AugAssign, _ast.AnnAssign, _ast.NamedExpr)):
                _target_names(n.target, assigned)
            elif isinstance(n, (_ast.For, _ast.AsyncFor)):      # (comprehension variables do not persist)
                _target_names(n.target, assigned)
            elif isinstance(n, (_ast.With, _ast.AsyncWith)):
                for it in n.items:
                    if it.optional_vars is not None:
                        _target_names(it.optional_vars, assigned)
            elif isinstance(n, _ast.Delete):
                for t in n.targets:
                    _target_names(t, assigned)
    for n in _ast.walk(loop.test):
        if isinstance(n, _ast.NamedExpr):
            _target_names(n.target, assigned)
    for part in [loop.test] + loop.body:
        for n in _ast.walk(part):
            if isinstance(n, _ast.Name) and isinstance(n.ctx, _ast.Load):
                read.add(n.id)
    return assigned, read


def _check_body(loop):
    def visit(node, in_loop):
        for c in _ast.iter_child_nodes(node):
            if isinstance(c, (_ast.FunctionDef, _ast.AsyncFunctionDef, _ast.Lambda, _ast.ClassDef)):
                continue
            if isinstance(c, (_ast.Return, _ast.Yield, _ast.YieldFrom, _ast.Await)) or (
                    not in_loop and isinstance(c, (_ast.Break, _ast.Continue))):
                raise MapError("line %d: %s inside a while-loop over rasters is not supported"
                               % (c.lineno, type(c).__name__.lower()))
            visit(c, in_loop or isinstance(c, (_ast.For, _ast.AsyncFor, _ast.While)))
    for stmt in loop.body:
        visit(_ast.Module(body=[stmt], type_ignores=[]), False)


def _swap_nodes(rasters):
    """Replaces, in place, the node of each raster by one holding its value
    (one evaluation for all)."""
    uniq = []
    seen = set()
    for r in rasters:
        if id(r) not in seen:
            seen.add(id(r))
            uniq.append(r)
    if not uniq:
        return
    n = len(uniq)
    arr = (Node * n)(*[r._node for r in uniq])
    out = (Node * n)()
    _lib.ma_materialize(arr, n, out)
    for r, m in zip(uniq, out):
        m = m.value if isinstance(m, Node) else m
        if m != r._node.value:
            tmp = Raster(Node(m))                      # a reference to the new node
            r._node, tmp._node = tmp._node, r._node
            del tmp                                    # releases the old one


class _Replay:
    """Answers raster truth requests while the test is replayed after the loop:
    the first one (the raster whose truth started the loop) with `first`, later
    ones with their evaluated truth; names read before the first request see
    their values from before the loop, as Python's own evaluation of the test
    did."""

    def __init__(self, first):
        self.first = first
        self.switched = False
        self.given = {}            # a raster asked again (the value of `a and b`) gets the same answer

    def answer(self, r):
        if id(r) in self.given:
            return self.given[id(r)][1]
        if not self.switched:
            self.switched = True
            v = self.first
        else:
            v = _truth_of(r)
        self.given[id(r)] = (r, v)
        return v


class _ReplayScope:
    def __init__(self, replay, before, lookup):
        self.replay, self.before, self.lookup = replay, before, lookup

    def __getitem__(self, name):
        if not self.replay.switched and name in self.before:
            return self.before[name]
        return self.lookup(name)


_loop_code = {}   # id(while statement) -> (statement, test code, body code, names assigned, names read)


def _compiled(loop, filename):
    c = _loop_code.get(id(loop))
    if c is None or c[0] is not loop:
        _check_body(loop)
        assigned, read = _loop_names(loop)
        c = (loop, compile(_ast.Expression(body=loop.test), filename, "eval"),
             compile(_ast.Module(body=loop.body, type_ignores=[]), filename, "exec"), assigned, read)
        if len(_loop_code) > 256:
            _loop_code.clear()
        _loop_code[id(loop)] = c
    return c


def _run_while(loop, frame):
    filename = frame.f_code.co_filename
    _, test_code, body_code, assigned, read = _compiled(loop, filename)
    g = frame.f_globals
    scope = frame.f_locals            # the module namespace at module level, else the frame's locals
    module_level = scope is g
    missing = object()
    # in a function, a name the body assigns that is not one of the function's
    # variables is declared global there: the body's stores go to its module
    # (a namespace frame, such as a module, a class body or an outer loop's
    # body, keeps its stores in its own mapping)
    co = frame.f_code
    own = set(co.co_varnames) | set(co.co_cellvars) | set(co.co_freevars)
    function = bool(co.co_flags & 0x1)   # CO_OPTIMIZED: the frame of a function
    to_module = {n for n in assigned if n not in own} if function and not module_level else set()

    def flush_globals():
        for n in to_module:
            try:
                if n in scope:
                    g[n] = scope[n]
                    del scope[n]
            except (KeyError, TypeError):
                pass

    def lookup(name):
        if name in scope:
            return scope[name]
        if name in g:
            return g[name]
        if hasattr(_builtins, name):
            return getattr(_builtins, name)
        raise KeyError(name)

    def get(name):
        try:
            return lookup(name)
        except KeyError:
            return missing

    test_names = {n.id for n in _ast.walk(loop.test) if isinstance(n, _ast.Name)}
    before = {n: get(n) for n in test_names}
    before = {k: v for k, v in before.items() if v is not missing}
    _swap_nodes([v for v in (get(n) for n in sorted(read - assigned)) if isinstance(v, Raster)])
    try:
        while True:
            _loop_tls.truth = getattr(_loop_tls, "truth", 0) + 1
            try:
                t = _builtins.eval(test_code, g, scope)
            finally:
                _loop_tls.truth -= 1
            carried = [v for v in (get(n) for n in sorted(assigned)) if isinstance(v, Raster)]
            if isinstance(t, Raster):
                if _lib.ma_numdim(t) != D0:
                    raise MapError("line %d: the while test is a 2-D raster: reduce it to a scalar (D0) raster first"
                                   % loop.test.lineno)
                _swap_nodes([t] + carried)
                go = bool(_lib.ma_value(t).value())
            else:
                _swap_nodes(carried)
                go = bool(t)
            del t, carried
            _lib.ma_collectGarbage()
            if not go:
                break
            _builtins.exec(body_code, g, scope)
            flush_globals()
    finally:
        flush_globals()
        if function and _sys.version_info < (3, 13):   # 3.13 frames' locals write through
            ct.pythonapi.PyFrame_LocalsToFast(ct.py_object(frame), ct.c_int(0))
    for first in (False, True):
        replay = _Replay(first)
        _loop_tls.replay = replay
        try:
            t = _builtins.eval(test_code, g, _ReplayScope(replay, before, lookup))
            if isinstance(t, Raster):            # the test itself: Python asks for its truth
                t = replay.answer(t)
        finally:
            _loop_tls.replay = None
        if not t:
            return first
    raise MapError("line %d: the while test stays true after the loop ended (a test with side effects?)"
                   % loop.test.lineno)


## Standalone functions


def setupDevices(plat_name, dev_type, dev_name):
    _lib.ma_setupDevices(plat_name.encode(), dev_type, dev_name.encode())


def eval(*args):
    # Note: shadows the built-in eval, as the reference module does
    cond = [isinstance(a, Raster) for a in args]
    if len(args) and not all(cond):
        if not any(cond):
            return _builtins.eval(*args)
        raise MapError("eval: mix of rasters and other arguments")
    num = len(args)
    NodeArr = Node * num
    nodearr = NodeArr(*[r._node for r in args])
    _lib.ma_eval(ct.cast(nodearr, ct.POINTER(Node)), num)


def value(arg):
    var = _lib.ma_value(arg)
    return var.value()


def read(file):
    return Raster(_lib.ma_read(os.fsencode(file)))


def write(raster, file):
    return _lib.ma_write(raster, os.fsencode(file))


def _cnst(cnst, ds, dt, mo, bs):
    var = Variant(cnst).convert(dt)
    return Raster(_lib.ma_constant(var, Array(ds), dt, mo, Array(bs)))


def zeros(ds=[], dt=F32, mo=ROW + BLK, bs=[]):
    return _cnst(0, ds, dt, mo, bs)


def ones(ds=[], dt=F32, mo=ROW + BLK, bs=[]):
    return _cnst(1, ds, dt, mo, bs)


def trues(ds=[], dt=B8, mo=ROW + BLK, bs=[]):
    return _cnst(True, ds, dt, mo, bs)


def falses(ds=[], dt=B8, mo=ROW + BLK, bs=[]):
    return _cnst(False, ds, dt, mo, bs)


def full(cnst, ds=[], dt=F32, mo=ROW + BLK, bs=[]):
    return _cnst(cnst, ds, dt, mo, bs)


def empty(ds=[], dt=F32, mo=ROW + BLK, bs=[]):
    return True


def _like(cnst, raster, dt, mo):
    dt = raster.datatype() if (dt == NONE_DATATYPE) else dt
    mo = raster.memorder() if (mo == NONE_MEMORDER) else mo
    var = Variant(cnst).convert(dt)
    ds = Array(raster.datasize())
    bs = Array(raster.blocksize())
    return Raster(_lib.ma_constant(var, ds, dt, mo, bs))


def zeros_like(raster, dt=NONE_DATATYPE, mo=NONE_MEMORDER):
    return _like(0, raster, dt, mo)


def ones_like(raster, dt=NONE_DATATYPE, mo=NONE_MEMORDER):
    return _like(1, raster, dt, mo)


def full_like(cnst, raster, dt=NONE_DATATYPE, mo=NONE_MEMORDER):
    return _like(cnst, raster, dt, mo)


def empty_like(raster, dt=NONE_DATATYPE, mo=NONE_MEMORDER):
    return True


def index(raster, dim):
    return Raster(_lib.ma_index(raster, dim))


def rand(seed, ds=[], dt=NONE_DATATYPE, mo=NONE_MEMORDER, bs=[]):
    ds = seed.datasize() if isinstance(seed, Raster) else ds
    dt = seed.datatype() if dt == NONE_DATATYPE else dt
    mo = BLK + ROW if mo == NONE_DATATYPE else mo
    bs = seed.blocksize() if isinstance(seed, Raster) else bs
    if not isinstance(seed, Raster):
        var = Variant(seed).convert(dt)
        seed = Raster(_lib.ma_constant(var, Array(ds), dt, mo, Array(bs)))
    return Raster(_lib.ma_rand(seed, dt, mo))


def astype(raster, dt):
    return Raster(_lib.ma_cast(raster, dt))


def con(cond, lhs, rhs):
    cond = _const_to_raster(cond)
    lhs = _const_to_raster(lhs)
    rhs = _const_to_raster(rhs)
    return Raster(_lib.ma_conditional(cond, lhs, rhs))


def _mask(lst):
    if not all(len(e) == len(lst[0]) for e in lst):
        raise MapError("mask rows differ in length")
    ds = Array([len(lst[0]), len(lst)])
    unroll = sum(lst, [])
    size = len(unroll)
    VarArr = Variant * size
    vararr = VarArr(*[Variant(e) for e in unroll])
    return ct.cast(vararr, ct.POINTER(Variant)), size, ds, vararr


def convolve(raster, lst):
    varptr, size, ds, _keep = _mask(lst)
    return Raster(_lib.ma_convolution(raster, varptr, size, ds))


def fsum(raster):
    lst = [[1, 1, 1], [1, 1, 1], [1, 1, 1]]
    return convolve(raster, lst)


def fmin(raster, lst):
    varptr, size, ds, _keep = _mask(lst)
    return Raster(_lib.ma_focalFunc(raster, varptr, size, ds, MIN))


def fmax(raster, lst):
    varptr, size, ds, _keep = _mask(lst)
    return Raster(_lib.ma_focalFunc(raster, varptr, size, ds, MAX))


# Focal percentages (front/Raster.cpp:437-448, no Python binding in the
# reference): the fraction of the mask-sized window around each cell whose
# cells the centre equals (percentage, AGE) or exceeds (percentile, ILE), in
# the raster's own type; the mask's values are not used, only its extent.
AGE, ILE = 1, 2


def percentage(raster, lst):
    varptr, size, ds, _keep = _mask(lst)
    return Raster(_lib.ma_focalPercent(raster, varptr, size, ds, AGE))


def percentile(raster, lst):
    varptr, size, ds, _keep = _mask(lst)
    return Raster(_lib.ma_focalPercent(raster, varptr, size, ds, ILE))


def zsum(raster):
    return Raster(_lib.ma_zonalReduc(raster, SUM))


def zprod(raster):
    return Raster(_lib.ma_zonalReduc(raster, PROD))


def zmax(raster):
    return Raster(_lib.ma_zonalReduc(raster, MAX))


def zmin(raster):
    return Raster(_lib.ma_zonalReduc(raster, MIN))


def rsum(raster, coord, radius=None):
    if radius:
        return Raster(_lib.ma_radialScanRadius(raster, SUM, Array(coord), float(radius)))
    return Raster(_lib.ma_radialScan(raster, SUM, Array(coord)))


def rprod(raster, coord, radius=None):
    if radius:
        return Raster(_lib.ma_radialScanRadius(raster, PROD, Array(coord), float(radius)))
    return Raster(_lib.ma_radialScan(raster, PROD, Array(coord)))


def rmax(raster, coord, radius=None):
    if radius:
        return Raster(_lib.ma_radialScanRadius(raster, MAX, Array(coord), float(radius)))
    return Raster(_lib.ma_radialScan(raster, MAX, Array(coord)))


def rmin(raster, coord, radius=None):
    if radius:
        return Raster(_lib.ma_radialScanRadius(raster, MIN, Array(coord), float(radius)))
    return Raster(_lib.ma_radialScan(raster, MIN, Array(coord)))


## Compound functions (python/map.py:592-706)

def lmax(lst):
    accu = lst[0]
    for i in range(1, len(lst)):
        accu = max(accu, lst[i])
    return accu


def lmin(lst):
    accu = lst[0]
    for i in range(1, len(lst)):
        accu = min(accu, lst[i])
    return accu


def lmaxpos(lst):
    maxim = lst[0]
    idx = zeros_like(maxim, U8)
    for i in range(1, len(lst)):
        idx = con(lst[i] > maxim, full_like(i, idx), idx)
        maxim = max(maxim, lst[i])
    return idx


def lminpos(lst):
    minim = lst[0]
    idx = zeros_like(minim, U8)
    for i in range(1, len(lst)):
        idx = con(lst[i] < minim, full_like(i, idx), idx)
        minim = min(minim, lst[i])
    return idx


def lor(lst):
    accu = lst[0]
    for i in range(1, len(lst)):
        accu = accu + lst[i]
    return accu


def pick(raster, lst):
    acu = _const_to_raster(lst[0])
    for i in range(len(lst)):
        acu = con(raster == i, lst[i], acu)
    return acu


def degrees(raster):
    return raster / (2 * PI) * 360


def radians(raster):
    return raster / 360 * (2 * PI)


PI = 3.141593


def distance(raster, coord):
    x = coord[0] - index(raster, D1)
    y = coord[1] - index(raster, D2)
    return sqrt(x * x + y * y + 0.0)


def mean(raster):
    return zsum(raster) / prod(raster.datasize())


def covariance(x, y):
    if x.datasize() != y.datasize():
        raise MapError("covariance: rasters differ in size")
    xydif = (x - mean(x)) * (y - mean(y))
    return zsum(xydif) / prod(x.datasize())


def gradient(raster):
    kx = [[-1, 0, 1], [-1, 0, 1], [-1, 0, 1]]
    ky = [[-1, -1, -1], [0, 0, 0], [1, 1, 1]]
    return convolve(raster, kx), convolve(raster, ky)


def blur(raster, size=3):
    if size == 3:
        krnl = [[1, 2, 1], [2, 4, 2], [1, 2, 1]]
        norm = 16
    elif size == 5:
        krnl = [[1, 4, 7, 4, 1], [4, 16, 26, 16, 4], [7, 26, 41, 26, 7], [4, 16, 26, 16, 4], [1, 4, 7, 4, 1]]
        norm = 276
    else:
        raise MapError("blur: size must be 3 or 5")
    return convolve(raster, krnl) / norm


def harris(raster):
    ix, iy = gradient(raster)
    xx, yy, xy = blur(ix * ix), blur(iy * iy), blur(ix * iy)
    return (xx * yy - xy) - 0.04 * (xx + yy) ** 2


def prod(arg):
    if isinstance(arg, (list, tuple)):
        return functools.reduce(operator.mul, arg, 1)
    elif isinstance(arg, Array):
        return arg.arr[0] * arg.arr[1]
    raise MapError("prod: unsupported argument")


## Extensions (no counterpart in the reference module)

_np_dtype = {F32: 'float32', F64: 'float64', B8: 'bool', U8: 'uint8', U16: 'uint16', U32: 'uint32',
             U64: 'uint64', S8: 'int8', S16: 'int16', S32: 'int32', S64: 'int64'}
_dt_of_np = {v: k for k, v in _np_dtype.items()}


def from_numpy(arr, bs=None, copy=True):
    """Raster input from a 2-D NumPy array (rows = y, columns = x)."""
    import numpy as np
    a = np.ascontiguousarray(arr)
    if a.ndim != 2:
        raise MapError("from_numpy: array must be 2-D")
    dt = _dt_of_np.get(a.dtype.name)
    if dt is None:
        raise MapError("from_numpy: unsupported dtype %s" % a.dtype)
    ds = Array([a.shape[1], a.shape[0]])
    node = _lib.ma_fromHost(a.ctypes.data_as(ct.c_void_p), ds, dt, Array(bs or []), 1 if copy else 0)
    r = Raster(node)
    if not copy:
        r._keep = a
    return r


def from_device(ptr, pitch, ds, dt, bs=None):
    """Raster input from device memory (pointer as int, pitch in bytes, ds = [x, y])."""
    return Raster(_lib.ma_fromDevice(ct.c_void_p(ptr), pitch, Array(ds), dt, Array(bs or [])))


def from_device_rows(ptr, pitch, ds, dt, row0, rows, bs=None):
    """Raster input from device memory holding only rows [row0, row0 + rows) of a
    ds = [x, y] raster (`ptr` is the address of row row0); evaluated by eval_rows."""
    return Raster(_lib.ma_fromDeviceRows(ct.c_void_p(ptr), pitch, Array(ds), dt, Array(bs or []), row0, rows))


def eval_rows(rasters, buffers, y0, y1):
    """Evaluates rows [y0, y1) of `rasters` into device buffers: buffers[i] =
    (address of row y0, pitch in bytes). Borders are decided in whole-raster
    coordinates, so the rows equal a whole-raster evaluation's."""
    n = len(rasters)
    dst = (ct.c_void_p * n)(*[b[0] for b in buffers])
    pitch = (ct.c_longlong * n)(*[b[1] for b in buffers])
    _lib.ma_evalRows(_node_array(rasters), n, dst, pitch, y0, y1)


def row_margin(*rasters):
    """Rows beyond a row range that eval_rows of these rasters reads from their inputs."""
    return _lib.ma_rowMargin(_node_array(rasters), len(rasters))


def bin_read_numpy(path):
    """The cells of a `.bin` file as a 2-D NumPy array (host only, no device)."""
    import numpy as np
    info = (ct.c_int * 7)()
    _lib.ma_binInfo(path.encode(), info)
    dt, _, w, h = info[0], info[1], info[2], info[3]
    out = np.empty((h, w), dtype=np.dtype(_np_dtype[dt]))
    _lib.ma_binReadHost(path.encode(), out.ctypes.data_as(ct.c_void_p), out.nbytes)
    return out


def bin_write_numpy(path, a, bs=(256, 256), mo=None):
    """Writes a 2-D NumPy array as a `.bin` file (ROW+BLK blocks of bs, or ROW)."""
    import numpy as np
    a = np.ascontiguousarray(a)
    dt = _dt_of_np[a.dtype.name]
    mo = ROW + BLK if mo is None else mo
    _lib.ma_binWriteHost(path.encode(), a.ctypes.data_as(ct.c_void_p), Array([a.shape[1], a.shape[0]]), dt, mo,
                         Array(list(bs)))


def to_numpy(raster, out=None):
    """Evaluates a raster and returns it as a 2-D NumPy array."""
    import numpy as np
    w, h = raster.datasize()
    dt = np.dtype(_np_dtype[raster.datatype()])
    if out is None:
        out = np.empty((h, w), dtype=dt)
    _lib.ma_toHost(raster, out.ctypes.data_as(ct.c_void_p), out.nbytes)
    return out


def to_device(raster, ptr, pitch, sync=True):
    _lib.ma_toDevice(raster, ct.c_void_p(ptr), pitch, 0 if sync else 1)


def materialize(*rasters):
    """Evaluates the rasters in one evaluation and returns, for each, a raster
    holding its value: 2-D results stay in device memory the library owns
    (released with the returned raster), scalars become constants."""
    out = []
    for r in rasters:
        c = Raster(r._node)
        out.append(c)
    _swap_nodes(out)
    return out


def node_count():
    """Nodes the runtime holds (after collect_garbage: the live ones)."""
    return _lib.ma_nodeCount()


def collect_garbage():
    """Drops the nodes no raster refers to, with the device memory they own."""
    _lib.ma_collectGarbage()


def set_border(mode):
    _lib.ma_setBorder(mode)


def get_border():
    return _lib.ma_getBorder()


def set_exec_mode(mode):
    _lib.ma_setExecMode(mode)


def get_exec_mode():
    return _lib.ma_getExecMode()


def set_stream_rows(rows):
    """Row bands of streamed host-to-host evaluation: 0 automatic, < 0 off, > 0 forced."""
    _lib.ma_setStreamRows(rows)


def get_stream_rows():
    return _lib.ma_getStreamRows()


def set_flow_jump_cells(cells):
    """Largest integer flow accumulation (cells) computed by pointer jumping;
    0 never, < 0 the default."""
    _lib.ma_setFlowJumpCells(int(cells))


def get_flow_jump_cells():
    return _lib.ma_getFlowJumpCells()


def set_paired_cells(on):
    """Two cells per thread step on packed f32x2 instructions in float focal groups
    (bit-identical results); False computes one cell at a time."""
    _lib.ma_setPairedCells(1 if on else 0)


def get_paired_cells():
    return bool(_lib.ma_getPairedCells())


def set_prediction(on):
    """Groups whose every output is one known value are filled without a launch."""
    _lib.ma_setPrediction(1 if on else 0)


def last_predicted_count():
    return _lib.ma_lastPredictedCount()


def set_algebraic_rewrite(on):
    """Hillshade compositions through the shading identity (no per-cell
    transcendental functions, results within the hillshade tolerance); False
    generates the literal operator chain; 2 the identity without its fast form."""
    _lib.ma_setAlgebraicRewrite(on if isinstance(on, int) and not isinstance(on, bool) else (1 if on else 0))


def get_algebraic_rewrite():
    return _lib.ma_getAlgebraicRewrite()


def last_band_count():
    return _lib.ma_lastBandCount()


def set_default_blocksize(bs):
    _lib.ma_setDefaultBlockSize(Array(bs))


def flow_direction(dem):
    """D8 steepest-descent direction codes (U8, 1 << dir in E,SE,S,SW,W,NW,N,NE order)."""
    return Raster(_lib.ma_focalFlow(dem))


def flow_accumulation(water, dirs):
    """Sum of `water` over every upstream cell along D8 directions (front/Raster.cpp:571-579)."""
    return Raster(_lib.ma_spreadScan(water, dirs, SUM))


def viewshed(dem, obs, h):
    """Height above the line of sight from observer `obs` at height `h` (front/Raster.cpp:558-569)."""
    shift = dem - h
    dist = distance(dem, obs)
    slope = shift / dist
    maxr = rmax(slope, obs)
    return (maxr * dist + h) - dem


def zonal_stats_device(value_ptr, value_pitch, zone_ptr, zone_pitch, W, H, nzones, count=0, vmin=0, vmax=0, sum=0,
                       mean=0, stream=None):
    """Per-zone statistics over device memory (pointers as ints, pitches in
    bytes); enqueued on `stream` (default: the library's stream), returns at
    once. Outputs are device arrays of `nzones` elements (0 to skip one)."""
    _lib.ma_zoneStats(ct.c_void_p(value_ptr), value_pitch, ct.c_void_p(zone_ptr), zone_pitch, W, H, nzones,
                      ct.c_void_p(count), ct.c_void_p(vmin), ct.c_void_p(vmax), ct.c_void_p(sum),
                      ct.c_void_p(mean), ct.c_void_p(_lib.ma_stream() if stream is None else stream))


def zonal_stats(value, zones, nzones):
    """Per-zone count / min / max / sum / mean of a float32 raster over an int32
    zone raster (a Raster or a 2-D NumPy array each). Cells with a zone id
    outside [0, nzones) or a NaN value are skipped. Returns a dict of NumPy
    arrays of `nzones` elements: count (uint64), min, max, sum, mean (float32)."""
    import numpy as np
    bufs = []

    def stage(x, dt, npdt):
        if isinstance(x, Raster):
            if x.datatype() != dt:
                raise MapError("zonal_stats: raster has datatype %s, %s expected" % (DataTypeId[x.datatype()],
                                                                                     DataTypeId[dt]))
            w, h = x.datasize()
            ptr = _lib.ma_devAlloc(max(1, w * h * 4))
            bufs.append(ptr)
            to_device(x, ptr, w * 4)
            return ptr, w, h
        a = np.ascontiguousarray(x, dtype=npdt)
        if a.ndim != 2:
            raise MapError("zonal_stats: arrays must be 2-D")
        ptr = _lib.ma_devAlloc(max(1, a.nbytes))
        bufs.append(ptr)
        if a.nbytes:
            _lib.ma_memcpy(ptr, a.ctypes.data_as(ct.c_void_p), a.nbytes, 1)
        return ptr, a.shape[1], a.shape[0]

    try:
        vp, w, h = stage(value, F32, np.float32)
        zp, zw, zh = stage(zones, S32, np.int32)
        if (w, h) != (zw, zh):
            raise MapError("zonal_stats: value and zone rasters differ in size")
        nz = int(nzones)
        out = _lib.ma_devAlloc(max(1, nz) * 24)
        bufs.append(out)
        zonal_stats_device(vp, w * 4, zp, w * 4, w, h, nz, out, out + 8 * nz, out + 12 * nz, out + 16 * nz,
                           out + 20 * nz)
        _lib.ma_sync()
        raw = np.empty(nz * 24, np.uint8)
        _lib.ma_memcpy(raw.ctypes.data_as(ct.c_void_p), out, raw.nbytes, 2)
        f = raw[8 * nz:].view(np.float32)
        return {"count": raw[:8 * nz].view(np.uint64).copy(), "min": f[:nz].copy(), "max": f[nz:2 * nz].copy(),
                "sum": f[2 * nz:3 * nz].copy(), "mean": f[3 * nz:].copy()}
    finally:
        for b in bufs:
            _lib.ma_devFree(b)


def sync():
    _lib.ma_sync()


def stream():
    return _lib.ma_stream()


def last_launch_count():
    return _lib.ma_lastLaunchCount()


def last_group_count():
    return _lib.ma_lastGroupCount()


def _node_array(rasters):
    NodeArr = Node * len(rasters)
    return NodeArr(*[r._node for r in rasters])


def describe_groups(*rasters):
    arr = _node_array(rasters)
    n = _lib.ma_describeGroups(arr, len(rasters), None, 0)
    buf = ct.create_string_buffer(n)
    _lib.ma_describeGroups(arr, len(rasters), buf, n)
    return buf.value.decode()


def generated_source(*rasters):
    arr = _node_array(rasters)
    n = _lib.ma_generatedSource(arr, len(rasters), None, 0)
    buf = ct.create_string_buffer(n)
    _lib.ma_generatedSource(arr, len(rasters), buf, n)
    return buf.value.decode()


def plain_schedule(*rasters):
    arr = _node_array(rasters)
    n = _lib.ma_plainSchedule(arr, len(rasters), None, 0)
    buf = ct.create_string_buffer(n)
    _lib.ma_plainSchedule(arr, len(rasters), buf, n)
    return [tuple(int(v) for v in line.split()) for line in buf.value.decode().splitlines() if line.strip()]


def compile_only(*rasters, compile=True):
    arr = _node_array(rasters)
    return _lib.ma_compileOnly(arr, len(rasters), 1 if compile else 0)


## CDLL interface: arguments & returns (python/map.py:723-830)

def _sig(name, argtypes, restype, check=True):
    f = getattr(_lib, name)
    f.argtypes = argtypes
    f.restype = restype
    if check:
        f.errcheck = _check


_lib.ma_errorCode.argtypes = []
_lib.ma_errorCode.restype = ct.c_int
_lib.ma_lastError.argtypes = []
_lib.ma_lastError.restype = ct.c_char_p

_sig('ma_setupDevices', [ct.c_char_p, ct.c_int, ct.c_char_p], None)
_sig('ma_increaseRef', [Raster], None)
_sig('ma_decreaseRef', [Raster], None, check=False)
_sig('ma_eval', [ct.POINTER(Node), ct.c_int], None)
_sig('ma_nodeid', [Raster], ct.c_int)
_sig('ma_streamdir', [Raster], ct.c_int)
_sig('ma_value', [Raster], Variant)
_sig('ma_datatype', [Raster], ct.c_int)
_sig('ma_numdim', [Raster], ct.c_int)
_sig('ma_memorder', [Raster], ct.c_int)
_sig('ma_datasize', [Raster], Array)
_sig('ma_blocksize', [Raster], Array)
_sig('ma_numblock', [Raster], Array)
_sig('ma_read', [ct.c_char_p], Node)
_sig('ma_write', [Raster, ct.c_char_p], ct.c_int)
_sig('ma_index', [Raster, ct.c_int], Node)
_sig('ma_rand', [Raster, ct.c_int, ct.c_int], Node)
_sig('ma_cast', [Raster, ct.c_int], Node)
_sig('ma_conditional', [Raster, Raster, Raster], Node)
_sig('ma_unary', [Raster, ct.c_int], Node)
_sig('ma_binary', [Raster, Raster, ct.c_int], Node)
_sig('ma_constant', [Variant, Array, ct.c_int, ct.c_int, Array], Node)
_sig('ma_access', [Raster, Array], Node)
_sig('ma_lhsAccess', [Raster, Raster, Array], Node)
_sig('ma_neighbor', [Raster, Array], Node)
_sig('ma_boundedNbh', [Raster, Raster, Raster], Node)
_sig('ma_convolution', [Raster, ct.POINTER(Variant), ct.c_int, Array], Node)
_sig('ma_focalFunc', [Raster, ct.POINTER(Variant), ct.c_int, Array, ct.c_int], Node)
_sig('ma_focalPercent', [Raster, ct.POINTER(Variant), ct.c_int, Array, ct.c_int], Node)
_sig('ma_zonalReduc', [Raster, ct.c_int], Node)
_sig('ma_radialScan', [Raster, ct.c_int, Array], Node)
_sig('ma_spreadScan', [Raster, Raster, ct.c_int], Node)
_sig('ma_radialScanRadius', [Raster, ct.c_int, Array, ct.c_double], Node)
_sig('ma_barrier', [Raster], Node)
_sig('ma_loopStart', [], None)
_sig('ma_loopCond', [Raster], None)
_sig('ma_loopBody', [], None)
_sig('ma_loopAgain', [], None)
_sig('ma_loopAssemble', [], Node)
_sig('ma_loopEnd', [], None)
_sig('ma_loopAgainTail', [Raster, ct.POINTER(ct.POINTER(Node)), ct.POINTER(ct.POINTER(Node)), ct.POINTER(ct.c_int)], None)
_sig('ma_setBorder', [ct.c_int], None)
_sig('ma_getBorder', [], ct.c_int, check=False)
_sig('ma_setExecMode', [ct.c_int], None)
_sig('ma_getExecMode', [], ct.c_int, check=False)
_sig('ma_setDefaultBlockSize', [Array], None)
_sig('ma_fromHost', [ct.c_void_p, Array, ct.c_int, Array, ct.c_int], Node)
_sig('ma_fromDevice', [ct.c_void_p, ct.c_longlong, Array, ct.c_int, Array], Node)
_sig('ma_toHost', [Raster, ct.c_void_p, ct.c_size_t], ct.c_int)
_sig('ma_toDevice', [Raster, ct.c_void_p, ct.c_longlong, ct.c_int], ct.c_int)
_sig('ma_materialize', [ct.POINTER(Node), ct.c_int, ct.POINTER(Node)], ct.c_int)
_sig('ma_collectGarbage', [], None)
_sig('ma_nodeCount', [], ct.c_int, check=False)
_sig('ma_sync', [], ct.c_int)
_sig('ma_stream', [], ct.c_void_p)
_sig('ma_lastLaunchCount', [], ct.c_int, check=False)
_sig('ma_lastGroupCount', [], ct.c_int, check=False)
_sig('ma_lastBandCount', [], ct.c_int, check=False)
_sig('ma_setStreamRows', [ct.c_int], None)
_sig('ma_getStreamRows', [], ct.c_int, check=False)
_sig('ma_setPairedCells', [ct.c_int], None)
_sig('ma_setFlowJumpCells', [ct.c_longlong], None)
_sig('ma_getFlowJumpCells', [], ct.c_longlong, check=False)
_sig('ma_getPairedCells', [], ct.c_int, check=False)
_sig('ma_setAlgebraicRewrite', [ct.c_int], None)
_sig('ma_setPrediction', [ct.c_int], None)
_sig('ma_binInfo', [ct.c_char_p, ct.POINTER(ct.c_int)], ct.c_int)
_sig('ma_binReadHost', [ct.c_char_p, ct.c_void_p, ct.c_size_t], ct.c_int)
_sig('ma_binWriteHost', [ct.c_char_p, ct.c_void_p, Array, ct.c_int, ct.c_int, Array], ct.c_int)
_sig('ma_getPrediction', [], ct.c_int, check=False)
_sig('ma_lastPredictedCount', [], ct.c_int, check=False)
_sig('ma_fromDeviceRows', [ct.c_void_p, ct.c_longlong, Array, ct.c_int, Array, ct.c_int, ct.c_int], Node)
_sig('ma_evalRows', [ct.POINTER(Node), ct.c_int, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_longlong), ct.c_int, ct.c_int],
     ct.c_int)
_sig('ma_rowMargin', [ct.POINTER(Node), ct.c_int], ct.c_int)
_sig('ma_getAlgebraicRewrite', [], ct.c_int, check=False)
_sig('ma_compileOnly', [ct.POINTER(Node), ct.c_int, ct.c_int], ct.c_int)
_sig('ma_describeGroups', [ct.POINTER(Node), ct.c_int, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_generatedSource', [ct.POINTER(Node), ct.c_int, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_plainSchedule', [ct.POINTER(Node), ct.c_int, ct.c_char_p, ct.c_size_t], ct.c_size_t)
if hasattr(_lib, 'ma_focalFlow'):
    _sig('ma_focalFlow', [Raster], Node)
_sig('ma_devAlloc', [ct.c_size_t], ct.c_void_p)
_sig('ma_zoneStats', [ct.c_void_p, ct.c_longlong, ct.c_void_p, ct.c_longlong, ct.c_int, ct.c_int, ct.c_int,
                      ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p], ct.c_int)
_sig('ma_devFree', [ct.c_void_p], None, check=False)
_sig('ma_hostAlloc', [ct.c_size_t], ct.c_void_p)
_sig('ma_hostFree', [ct.c_void_p], None, check=False)
_sig('ma_memcpy', [ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_int], ct.c_int)
_sig('ma_evalAsync', [ct.POINTER(Node), ct.c_int], ct.c_int)
_sig('ma_totalLaunchCount', [], ct.c_int, check=False)
_sig('ma_setDevice', [ct.c_int], None)


class Batch:
    """Batched persistent execution of many programs (see ma_batchAdd).

    add(outputs, buffers) registers one program: `outputs` are rasters and
    `buffers` (device pointer, pitch in bytes) receive them. run() launches
    every registered program as one persistent kernel per dependency level."""

    def __init__(self):
        self._h = _lib.ma_batchCreate()
        self._keep = []

    def add(self, outputs, buffers):
        n = len(outputs)
        arr = _node_array(outputs)
        dst = (ct.c_void_p * n)(*[b[0] for b in buffers])
        pitch = (ct.c_longlong * n)(*[b[1] for b in buffers])
        self._keep.append(outputs)
        return _lib.ma_batchAdd(self._h, arr, n, dst, pitch)

    def prepare(self, autotune=True):
        _lib.ma_batchPrepare(self._h, 1 if autotune else 0)

    def run(self, sync=True):
        _lib.ma_batchRun(self._h, 1 if sync else 0)

    def info(self):
        import json
        n = _lib.ma_batchInfo(self._h, None, 0)
        buf = ct.create_string_buffer(n)
        _lib.ma_batchInfo(self._h, buf, n)
        return json.loads(buf.value.decode())

    def __del__(self):
        try:
            if self._h:
                _lib.ma_batchDestroy(self._h)
                self._h = None
        except Exception:
            pass


_sig('ma_batchCreate', [], ct.c_void_p)
_sig('ma_batchAdd', [ct.c_void_p, ct.POINTER(Node), ct.c_int, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_longlong)], ct.c_int)
_sig('ma_batchPrepare', [ct.c_void_p, ct.c_int], ct.c_int)
_sig('ma_batchRun', [ct.c_void_p, ct.c_int], ct.c_int)
_sig('ma_batchInfo', [ct.c_void_p, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_batchDestroy', [ct.c_void_p], None, check=False)


class Server:
    """Serving over a device-resident DEM with continuous batching (ma_server*)."""
    HILLSHADE, SLOPE, VIEWSHED, FLOW = 0, 1, 2, 3

    def __init__(self, dem_ptr, pitch, width, height, budget_bytes, max_batch=256):
        self._h = _lib.ma_serverCreate(ct.c_void_p(dem_ptr), pitch, width, height, budget_bytes, max_batch)

    def submit(self, kind, x0, y0, w, h, obs=(0, 0), obs_h=10.0, radius=0.0):
        return _lib.ma_serverSubmit(self._h, kind, x0, y0, w, h, obs[0], obs[1], obs_h, radius)

    def wait(self, rid, timeout=-1.0):
        return _lib.ma_serverWait(self._h, rid, timeout)

    def result(self, rid, shape, dtype):
        import numpy as np
        out = np.empty(shape, dtype=dtype)
        _lib.ma_serverResult(self._h, rid, out.ctypes.data_as(ct.c_void_p), out.nbytes)
        return out

    def release(self, rid):
        _lib.ma_serverRelease(self._h, rid)

    def latency_ms(self, rid):
        return _lib.ma_serverLatency(self._h, rid)

    def stats(self):
        import json
        n = _lib.ma_serverStats(self._h, None, 0)
        buf = ct.create_string_buffer(n)
        _lib.ma_serverStats(self._h, buf, n)
        return json.loads(buf.value.decode())

    def load(self, rate, seconds, mix=(0.5, 0.2, 0.15, 0.15), seed=0, obs_h=10.0, radius=167.0):
        import json
        m = (ct.c_double * 4)(*mix)
        cap = 1 << 16
        buf = ct.create_string_buffer(cap)
        n = _lib.ma_serverLoad(self._h, rate, seconds, m, seed, obs_h, radius, buf, cap)
        return json.loads(buf.value.decode())

    def load_closed(self, outstanding, seconds, mix=(0.5, 0.2, 0.15, 0.15), seed=0, obs_h=10.0, radius=167.0):
        """Closed loop: `outstanding` requests in flight for `seconds`."""
        import json
        m = (ct.c_double * 4)(*mix)
        cap = 1 << 16
        buf = ct.create_string_buffer(cap)
        _lib.ma_serverLoadClosed(self._h, outstanding, seconds, m, seed, obs_h, radius, buf, cap)
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            _lib.ma_serverDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_sig('ma_serverCreate', [ct.c_void_p, ct.c_longlong, ct.c_int, ct.c_int, ct.c_size_t, ct.c_int], ct.c_void_p)
_sig('ma_serverSubmit', [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_float,
                         ct.c_double], ct.c_longlong)
_sig('ma_serverWait', [ct.c_void_p, ct.c_longlong, ct.c_double], ct.c_int)
_sig('ma_serverResult', [ct.c_void_p, ct.c_longlong, ct.c_void_p, ct.c_size_t], ct.c_int)
_sig('ma_serverRelease', [ct.c_void_p, ct.c_longlong], ct.c_int)
_sig('ma_serverLatency', [ct.c_void_p, ct.c_longlong], ct.c_double)
_sig('ma_serverStats', [ct.c_void_p, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_serverLoad', [ct.c_void_p, ct.c_double, ct.c_double, ct.POINTER(ct.c_double), ct.c_uint, ct.c_double,
                       ct.c_double, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_serverLoadClosed', [ct.c_void_p, ct.c_int, ct.c_double, ct.POINTER(ct.c_double), ct.c_uint, ct.c_double,
                             ct.c_double, ct.c_char_p, ct.c_size_t], ct.c_size_t)
_sig('ma_serverDestroy', [ct.c_void_p], None)
