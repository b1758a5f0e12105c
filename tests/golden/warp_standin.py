"""A small pure-Python stand-in for the NVIDIA Warp API that
mmichelis/WarpVBD ``src/vbd_solver.py`` uses -- TEST INFRASTRUCTURE ONLY.

warp-lang 1.10.0 (the reference's pinned dependency, ``environment.yml:9``)
cannot be installed offline, so the reference solver cannot run on its own
runtime here.  Registered as ``sys.modules['warp']``, this module lets the
reference's ``vbd_solver.py`` execute *unchanged* on the CPU, one kernel
thread after another, so that its own time step can produce golden
trajectories (``make_ref_trajectories.py``).  Nothing outside
``tests/golden`` imports it.

What is restated, from Warp's published semantics:

* ``@wp.kernel`` / ``@wp.func``: plain Python functions; ``wp.launch`` calls
  the kernel once per thread index of ``dim`` (row-major over a 2-D ``dim``),
  ``wp.tid()`` returns that index; ``wp.launch_tiled`` calls it once per tile
  (``wp.tid()`` = tile index), the tile operations acting on whole tiles.
* ``vec3d`` / ``vec4i`` / ``mat33d`` value types: component-wise ``+ - /``,
  scalar scaling, ``mat * mat`` and ``mat * vec`` as matrix products (Warp's
  ``*`` between matrices), ``m[i, j]`` and ``m[i]`` (a row) indexing.
* ``determinant`` (row0 . (row1 x row2)), ``inverse`` (adjugate / det, a zero
  matrix when det == 0), ``transpose``, ``trace``, ``identity``,
  ``matrix_from_cols``.
* arrays of scalars / vectors / matrices over NumPy storage with the trailing
  vector or matrix dimensions, element and sub-array indexing, ``numpy()``,
  ``clone``, ``zeros``, ``zeros_like``, ``ones``, and the elementwise ``-`` and
  ``/`` the reference applies to whole arrays (``vbd_solver.py:609``).
* tiles: ``tile_load`` pads the rows past the source array with zeros (Warp's
  out-of-bounds tile semantics, relied on at ``vbd_solver.py:260-261`` where
  32 rows are loaded from a 20-row slice), ``tile_sum`` adds the rows in
  order, ``tile_cholesky`` is the Cholesky-Banachiewicz factorisation (a
  non-positive pivot gives NaN, as a square root of a negative number does),
  ``tile_cholesky_solve`` forward and back substitution, ``tile_store``.

All arithmetic is IEEE double precision (Python floats), as in the reference,
whose types are all ``float64``.  The order of the additions inside a matrix
product, a determinant or a tile sum may differ from Warp's compiled code in
the last bit; over a trajectory that is far below the tolerances the tests
apply.
"""
import itertools
import math

import numpy as np

# ---------------------------------------------------------------------------
# scalar types: constructors that double as dtype markers
# ---------------------------------------------------------------------------


class _Scalar:
    def __init__(self, name, conv, np_dtype):
        self.__name__ = name
        self._conv = conv
        self.np_dtype = np_dtype
        self.elem_shape = ()

    def __call__(self, x=0):
        return self._conv(x)

    def __repr__(self):
        return f"warp_standin.{self.__name__}"


float64 = _Scalar("float64", float, np.float64)
float32 = _Scalar("float32", float, np.float64)  # unused by the solver; kept in fp64
int32 = _Scalar("int32", int, np.int32)
bool = _Scalar("bool", lambda x: x if isinstance(x, type(True)) else x != 0, np.bool_)  # noqa: A001


def _is_scalar(x):
    return isinstance(x, (int, float, np.floating, np.integer))


# ---------------------------------------------------------------------------
# vector and matrix value types
# ---------------------------------------------------------------------------


class _VecBase:
    __slots__ = ("v",)
    n = 3
    conv = float

    def __init__(self, *args):
        if not args:
            self.v = [self.conv(0)] * self.n
        elif len(args) == 1:
            self.v = [self.conv(a) for a in args[0]]
        else:
            self.v = [self.conv(a) for a in args]
        if len(self.v) != self.n:
            raise ValueError(f"{type(self).__name__} takes {self.n} components")

    def _new(self, vals):
        o = object.__new__(type(self))
        o.v = vals
        return o

    def __getitem__(self, i):
        return self.v[i]

    def __setitem__(self, i, x):
        self.v[i] = self.conv(x)

    def __iter__(self):
        return iter(self.v)

    def __len__(self):
        return self.n

    def __add__(self, o):
        return self._new([a + b for a, b in zip(self.v, o.v)])

    def __sub__(self, o):
        return self._new([a - b for a, b in zip(self.v, o.v)])

    def __neg__(self):
        return self._new([-a for a in self.v])

    def __mul__(self, s):
        if _is_scalar(s):
            return self._new([a * s for a in self.v])
        return NotImplemented

    def __rmul__(self, s):
        if _is_scalar(s):
            return self._new([s * a for a in self.v])
        return NotImplemented

    def __truediv__(self, s):
        return self._new([a / s for a in self.v])

    def __repr__(self):
        return f"{type(self).__name__}({', '.join(map(repr, self.v))})"


class vec3d(_VecBase):  # noqa: N801 (Warp's name)
    __slots__ = ()
    n = 3
    conv = float
    elem_shape = (3,)
    np_dtype = np.float64


class vec4i(_VecBase):  # noqa: N801
    __slots__ = ()
    n = 4
    conv = int
    elem_shape = (4,)
    np_dtype = np.int32


class mat33d:  # noqa: N801
    """3x3 float64 matrix, row-major list of 9 values."""
    __slots__ = ("m",)
    elem_shape = (3, 3)
    np_dtype = np.float64

    def __init__(self, *args):
        if not args:
            self.m = [0.0] * 9
        elif len(args) == 9:
            self.m = [float(a) for a in args]
        else:
            a = np.asarray(args[0], dtype=np.float64).reshape(9)
            self.m = [float(x) for x in a]

    @staticmethod
    def _of(vals):
        o = object.__new__(mat33d)
        o.m = vals
        return o

    def __getitem__(self, idx):
        if isinstance(idx, tuple):
            r, c = idx
            return self.m[3 * r + c]
        return vec3d(self.m[3 * idx:3 * idx + 3])

    def __setitem__(self, idx, x):
        r, c = idx
        self.m[3 * r + c] = float(x)

    def __add__(self, o):
        return mat33d._of([a + b for a, b in zip(self.m, o.m)])

    def __sub__(self, o):
        return mat33d._of([a - b for a, b in zip(self.m, o.m)])

    def __neg__(self):
        return mat33d._of([-a for a in self.m])

    def __mul__(self, o):
        if _is_scalar(o):
            return mat33d._of([a * o for a in self.m])
        a = self.m
        if isinstance(o, mat33d):
            b = o.m
            return mat33d._of([a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c]
                               for r in range(3) for c in range(3)])
        if isinstance(o, vec3d):
            x = o.v
            return vec3d._of_list([a[3 * r] * x[0] + a[3 * r + 1] * x[1] + a[3 * r + 2] * x[2]
                                   for r in range(3)])
        return NotImplemented

    def __rmul__(self, s):
        if _is_scalar(s):
            return mat33d._of([s * a for a in self.m])
        return NotImplemented

    def __truediv__(self, s):
        return mat33d._of([a / s for a in self.m])

    def tolist(self):
        return [self.m[0:3], self.m[3:6], self.m[6:9]]

    def __repr__(self):
        return f"mat33d({self.tolist()})"


def _vec3_of_list(vals):
    o = object.__new__(vec3d)
    o.v = vals
    return o


vec3d._of_list = staticmethod(_vec3_of_list)


# ---------------------------------------------------------------------------
# builtins
# ---------------------------------------------------------------------------


def abs(x):  # noqa: A001 (Warp's name)
    return -x if x < 0 else x


def identity(n=3, dtype=float64):
    if n != 3:
        raise NotImplementedError("only 3x3")
    return mat33d(1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)


def transpose(a):
    m = a.m
    return mat33d._of([m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]])


def trace(a):
    m = a.m
    return m[0] + m[4] + m[8]


def determinant(a):
    m = a.m
    # row0 . (row1 x row2)
    cx = m[4] * m[8] - m[5] * m[7]
    cy = m[5] * m[6] - m[3] * m[8]
    cz = m[3] * m[7] - m[4] * m[6]
    return m[0] * cx + m[1] * cy + m[2] * cz


def inverse(a):
    m = a.m
    det = determinant(a)
    if det == 0.0:
        return mat33d()
    adj = [m[4] * m[8] - m[5] * m[7], m[2] * m[7] - m[1] * m[8], m[1] * m[5] - m[2] * m[4],
           m[5] * m[6] - m[3] * m[8], m[0] * m[8] - m[2] * m[6], m[2] * m[3] - m[0] * m[5],
           m[3] * m[7] - m[4] * m[6], m[1] * m[6] - m[0] * m[7], m[0] * m[4] - m[1] * m[3]]
    s = 1.0 / det
    return mat33d._of([x * s for x in adj])


def matrix_from_cols(c0, c1, c2):
    a, b, c = c0.v, c1.v, c2.v
    return mat33d._of([a[0], b[0], c[0], a[1], b[1], c[1], a[2], b[2], c[2]])


# ---------------------------------------------------------------------------
# arrays
# ---------------------------------------------------------------------------


def _elem_shape(dtype):
    return getattr(dtype, "elem_shape", ())


def _np_dtype(dtype):
    return getattr(dtype, "np_dtype", np.float64)


class array:  # noqa: N801
    """Array of scalars, vectors or matrices over NumPy storage whose
    trailing dimensions are the element's.  Without data it is only a type
    annotation (``wp.array(dtype=wp.vec3d)`` in a kernel signature)."""

    def __init__(self, data=None, dtype=float64, shape=None, device=None, ndim=None,
                 _storage=None, **_):
        self.dtype = dtype
        self.device = device
        if _storage is not None:
            self._s = _storage
        elif data is None:
            self._s = None if shape is None else np.zeros(
                (tuple(shape) if not isinstance(shape, int) else (shape,)) + _elem_shape(dtype),
                dtype=_np_dtype(dtype))
        else:
            src = data._s if isinstance(data, array) else np.asarray(data)
            self._s = np.array(src, dtype=_np_dtype(dtype), copy=True)
            es = _elem_shape(dtype)
            if es and tuple(self._s.shape[-len(es):]) != es:
                self._s = self._s.reshape(self._s.shape[:-1] + es) if es == (3, 3) else self._s
        self._nd = None if self._s is None else self._s.ndim - len(_elem_shape(dtype))

    @property
    def shape(self):
        es = len(_elem_shape(self.dtype))
        return self._s.shape[:self._s.ndim - es]

    @property
    def ndim(self):
        return self._nd

    def numpy(self):
        return self._s

    def _box(self, raw):
        d = self.dtype
        if d is vec3d:
            return _vec3_of_list(raw.tolist())
        if d is mat33d:
            return mat33d._of(raw.reshape(9).tolist())
        if d is vec4i:
            o = object.__new__(vec4i)
            o.v = raw.tolist()
            return o
        return raw.item()

    def __getitem__(self, idx):
        t = idx if isinstance(idx, tuple) else (idx,)
        if len(t) == self._nd:
            return self._box(self._s[t])
        return array(dtype=self.dtype, device=self.device, _storage=self._s[t])

    def __setitem__(self, idx, value):
        t = idx if isinstance(idx, tuple) else (idx,)
        if isinstance(value, _VecBase):
            value = value.v
        elif isinstance(value, mat33d):
            value = value.tolist()
        self._s[t] = value

    def __len__(self):
        return self._s.shape[0]

    # whole-array arithmetic (vbd_solver.py:609)
    def __sub__(self, o):
        return array(dtype=self.dtype, device=self.device, _storage=self._s - o._s)

    def __add__(self, o):
        return array(dtype=self.dtype, device=self.device, _storage=self._s + o._s)

    def __truediv__(self, s):
        return array(dtype=self.dtype, device=self.device, _storage=self._s / float(s))


def array2d(dtype=float64, **kw):
    return array(dtype=dtype, **kw)


array3d = array4d = array2d


def zeros(shape=None, dtype=float64, device=None, **_):
    return array(dtype=dtype, shape=shape, device=device)


def zeros_like(a):
    return array(dtype=a.dtype, device=a.device, _storage=np.zeros_like(a._s))


def ones(shape, dtype=float64, device=None, **_):
    a = zeros(shape, dtype, device)
    a._s[...] = 1
    return a


def clone(a, device=None):
    return array(dtype=a.dtype, device=a.device, _storage=a._s.copy())


# ---------------------------------------------------------------------------
# kernels and launches
# ---------------------------------------------------------------------------

_tid = [0]
launch_counts = {}  # kernel name -> launches so far (the generator reads sweep counts off it)


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.key = fn.__name__


def kernel(fn=None, **_):
    if fn is None:
        return lambda f: Kernel(f)
    return Kernel(fn)


def func(fn=None, **_):
    if fn is None:
        return lambda f: f
    return fn


def tid():
    return _tid[0]


def _run(kern, dims, args):
    launch_counts[kern.key] = launch_counts.get(kern.key, 0) + 1
    fn = kern.fn
    if len(dims) == 1:
        for i in range(dims[0]):
            _tid[0] = i
            fn(*args)
    else:
        for t in itertools.product(*(range(d) for d in dims)):
            _tid[0] = t
            fn(*args)


def launch(kernel, dim, inputs=(), outputs=(), device=None, **_):
    dims = (dim,) if isinstance(dim, int) else tuple(int(d) for d in dim)
    _run(kernel, dims, list(inputs) + list(outputs))


def launch_tiled(kernel, dim, inputs=(), outputs=(), block_dim=None, device=None, **_):
    dims = (dim,) if isinstance(dim, int) else tuple(int(d) for d in dim)
    _run(kernel, dims, list(inputs) + list(outputs))


def synchronize_device(device=None):
    pass


def synchronize():
    pass


# ---------------------------------------------------------------------------
# tiles (one tile per launch_tiled index)
# ---------------------------------------------------------------------------


def tile_load(a, shape, offset=None, **_):
    src = a._s
    out = np.zeros(tuple(shape), dtype=src.dtype)
    n = min(src.shape[0], out.shape[0])
    out[:n] = src[:n]
    return out


def tile_sum(t, axis=None):
    if axis is None:
        acc = 0.0
        for x in t.reshape(-1):
            acc = acc + float(x)
        return np.array([acc])
    if axis != 0:
        raise NotImplementedError("tile_sum over axis 0 only")
    acc = t[0].copy()
    for r in range(1, t.shape[0]):
        acc = acc + t[r]
    return acc


def _sqrt(x):
    return math.sqrt(x) if x >= 0.0 else float("nan")


def tile_cholesky(A):
    A = np.asarray(A, dtype=np.float64)
    n = A.shape[0]
    L = np.zeros_like(A)
    for i in range(n):
        for j in range(i + 1):
            s = float(A[i, j])
            for k in range(j):
                s -= float(L[i, k]) * float(L[j, k])
            L[i, j] = _sqrt(s) if i == j else s / float(L[j, j])
    return L


def tile_cholesky_solve(L, b):
    L = np.asarray(L, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = L.shape[0]
    y = np.zeros(n)
    for i in range(n):
        s = float(b[i])
        for k in range(i):
            s -= float(L[i, k]) * float(y[k])
        y[i] = s / float(L[i, i])
    x = np.zeros(n)
    for i in reversed(range(n)):
        s = float(y[i])
        for k in range(i + 1, n):
            s -= float(L[k, i]) * float(x[k])
        x[i] = s / float(L[i, i])
    return x


def tile_store(dst, t, offset=None, **_):
    dst._s[...] = t


class ScopedDevice:
    def __init__(self, device=None):
        self.device = device

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def init():
    pass
