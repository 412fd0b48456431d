"""ctypes front end to the parity oracle (TEST INFRASTRUCTURE).

Two CPU implementations of KORAL's hot path are reachable from here:

* ``OracleGrid`` drives the C restatement in ``koral_oracle.c`` (run-time grid
  size and scheme), built by ``oracle/Makefile`` into
  ``oracle/_ref/libkoral_oracle.so``;
* ``RefKoral`` drives the reference KORAL sources themselves, compiled per
  problem by ``oracle/ref/build_ref.sh`` into ``oracle/_ref/libkref_*.so``;
* ``RefRadCells`` calls the reference's per-cell radiation routines (M1
  closure, implicit source solve) on independent cells of the radiating-cells
  build.

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this module; the product never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_LIB = os.path.join(REF_DIR, "libkoral_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _i(a):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def _lib(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built")
    return ctypes.CDLL(path)


class OracleGrid:
    """One grid of the C restatement oracle."""

    ARR = dict(u=0, p=1, g=2, G=3, gKr=4, gbx=5, gby=6, gbz=7, Gbx=8, Gby=9, Gbz=10,
               flbx=11, flby=12, flbz=13, xbx=14, xby=15, xbz=16, xcx=17, xcy=18, xcz=19, emf=20)

    _lib_handle = None

    @classmethod
    def lib(cls):
        if cls._lib_handle is None:
            L = _lib(ORACLE_LIB)
            L.ko_grid_create.restype = ctypes.c_void_p
            L.ko_grid_create.argtypes = [ctypes.c_int] * 6
            L.ko_grid_destroy.argtypes = [ctypes.c_void_p]
            L.ko_array.restype = _dp
            L.ko_array.argtypes = [ctypes.c_void_p, ctypes.c_int]
            L.ko_scalar.restype = ctypes.c_double
            L.ko_scalar.argtypes = [ctypes.c_void_p, ctypes.c_int]
            L.ko_set_scalar.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
            L.ko_set_physics.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
            L.ko_set_floors.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 5
            L.ko_set_uniform_grid.argtypes = [ctypes.c_void_p, _dp, _dp]
            L.ko_layout.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
            for fn in ("ko_set_minkowski_metric", "ko_set_bc", "ko_calc_wavespeeds", "ko_calc_u2p",
                       "ko_save_timesteps", "ko_begin_run", "ko_init_orszag_tang"):
                getattr(L, fn).argtypes = [ctypes.c_void_p]
            L.ko_begin_step.argtypes = [ctypes.c_void_p]
            L.ko_begin_step.restype = ctypes.c_double
            L.ko_rk2_step.argtypes = [ctypes.c_void_p]
            L.ko_op_explicit.argtypes = [ctypes.c_void_p, ctypes.c_double]
            ip = ctypes.POINTER(ctypes.c_int)
            L.ko_u2p_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, ip, ip]
            L.ko_p2u_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp]
            L.ko_floors_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, ip]
            cls._lib_handle = L
        return cls._lib_handle

    def __init__(self, nx, ny, nz, ng, nv=9, axisym=0):
        self.L = self.lib()
        self.h = self.L.ko_grid_create(nx, ny, nz, ng, nv, axisym)
        lay = (ctypes.c_int * 16)()
        self.L.ko_layout(self.h, lay)
        self.nx, self.ny, self.nz, self.ng, self.nv, self.sx, self.sy, self.sz, self.szmet = lay[:9]

    def close(self):
        if self.h:
            self.L.ko_grid_destroy(self.h)
            self.h = None

    __del__ = close

    def array(self, name):
        ptr = self.L.ko_array(self.h, self.ARR[name])
        if name in ("u", "p"):
            shape = (self.sz, self.sy, self.sx, self.nv)
        else:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=shape)

    def scalar(self, i):
        return self.L.ko_scalar(self.h, i)

    def u2p_batch(self, uu, pp, g, G):
        """Per-cell u2p (u2p.c:176) on n independent cells; returns (pp, status, fixup)."""
        uu = np.ascontiguousarray(uu, dtype=np.float64)
        pp = np.ascontiguousarray(pp, dtype=np.float64).copy()
        g = np.ascontiguousarray(g, dtype=np.float64)
        G = np.ascontiguousarray(G, dtype=np.float64)
        n = uu.shape[0]
        st = np.zeros(n, dtype=np.int32)
        fx = np.zeros(n, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self.L.ko_u2p_batch(self.h, n, uu.ctypes.data_as(_dp), pp.ctypes.data_as(_dp), g.ctypes.data_as(_dp),
                            G.ctypes.data_as(_dp), st.ctypes.data_as(ip), fx.ctypes.data_as(ip))
        return pp, st, fx

    def p2u_batch(self, pp, g, G):
        pp = np.ascontiguousarray(pp, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        G = np.ascontiguousarray(G, dtype=np.float64)
        uu = np.empty_like(pp)
        self.L.ko_p2u_batch(self.h, pp.shape[0], pp.ctypes.data_as(_dp), uu.ctypes.data_as(_dp),
                            g.ctypes.data_as(_dp), G.ctypes.data_as(_dp))
        return uu

    def set_physics(self, gamma, tsteplim, int_order, fluxmethod):
        self.L.ko_set_physics(self.h, gamma, tsteplim, int_order, fluxmethod)

    def set_floors(self, rhofloor, uurhomin, uurhomax, b2rhomax, gammamax):
        self.L.ko_set_floors(self.h, rhofloor, uurhomin, uurhomax, b2rhomax, gammamax)

    def set_uniform_grid(self, lo, hi):
        lo = (ctypes.c_double * 3)(*lo)
        hi = (ctypes.c_double * 3)(*hi)
        self.L.ko_set_uniform_grid(self.h, lo, hi)

    def __getattr__(self, name):
        fn = getattr(self.lib(), "ko_" + name)
        return lambda *a: fn(self.h, *a)


def orszag_tang_oracle(n=128):
    """Relativistic Orszag-Tang vortex on an n x n periodic grid, set up
    exactly as the reference plug-in oracle/ref/problems/ORSZAGREL does."""
    G = OracleGrid(n, n, 1, 3, 9)
    G.set_physics(5.0 / 3.0, 0.5, 2, 0)
    G.set_uniform_grid([0.0, 0.0, -1.0], [2 * np.pi, 2 * np.pi, 1.0])
    G.set_minkowski_metric()
    G.init_orszag_tang()
    G.begin_run()
    return G


class RefKoral:
    """The reference KORAL build for one problem (compile-time grid)."""

    def __init__(self, libname):
        path = os.path.join(REF_DIR, libname)
        self.L = _lib(path)
        sz = (ctypes.c_int * 16)()
        self.L.kref_sizes(sz)
        (self.nx, self.ny, self.nz, self.ng, self.nv, self.sx, self.sy, self.sz, self.szmet,
         self.int_order, self.fluxmethod, self.timestepping, self.magn, self.rad, self.coords) = sz[:15]
        self.L.kref_begin_step.restype = ctypes.c_double
        self.L.op_explicit.argtypes = [ctypes.c_double, ctypes.c_double]
        self.L.op_implicit.argtypes = [ctypes.c_double, ctypes.c_double]

    def init(self):
        self.L.kref_init()

    def step(self, n=1):
        return self.L.kref_nsteps(n)

    def array(self, name, shape=None):
        ptr = _dp.in_dll(self.L, name)
        if shape is None:
            shape = (self.sz, self.sy, self.sx, self.nv)
        return np.ctypeslib.as_array(ptr, shape=shape)

    def scalar(self, name):
        return ctypes.c_double.in_dll(self.L, name).value

    def physics(self):
        out = (ctypes.c_double * 16)()
        self.L.kref_physics(out)
        keys = ("gamma", "tsteplim", "rhofloor", "uurhoratiomin", "uurhoratiomax", "b2rhoratiomax",
                "gammamaxhd", "u2pconv", "spin", "axisym")
        return dict(zip(keys, out[:10]))

    def grid_faces(self):
        """Cell-face coordinates per axis, xb[ic+NG] for ic in [-NG, N+NG]."""
        n = (self.nx, self.ny, self.nz)
        tot = sum(k + 1 + 2 * self.ng for k in n)
        xb = np.ctypeslib.as_array(_dp.in_dll(self.L, "xb"), shape=(tot,)).copy()
        out, o = [], 0
        for k in n:
            out.append(xb[o:o + k + 1 + 2 * self.ng])
            o += k + 1 + 2 * self.ng
        return out

    def metric_tables(self):
        """(g, G, gKr, gbx, gby, gbz, Gbx, Gby, Gbz) in KORAL layout."""
        sx, sy, sm = self.sx, self.sy, self.szmet
        sizes = dict(g=sx * sy * sm * 20, G=sx * sy * sm * 20, gKr=sx * sy * sm * 64,
                     gbx=(sx + 1) * sy * sm * 20, Gbx=(sx + 1) * sy * sm * 20,
                     gby=sx * (sy + 1) * sm * 20, Gby=sx * (sy + 1) * sm * 20,
                     gbz=sx * sy * (sm + 1) * 20, Gbz=sx * sy * (sm + 1) * 20)
        return tuple(np.ctypeslib.as_array(_dp.in_dll(self.L, k), shape=(sizes[k],)).copy()
                     for k in ("g", "G", "gKr", "gbx", "gby", "gbz", "Gbx", "Gby", "Gbz"))

    def rhofloor_table(self):
        c = np.zeros(self.sx)
        f = np.zeros(self.sx + 1)
        ok = self.L.kref_rhofloor_table(c.ctypes.data_as(_dp), f.ctypes.data_as(_dp))
        return (c, f) if ok else (None, None)

    def set_scalar(self, name, v):
        ctypes.c_double.in_dll(self.L, name).value = v


class RefRadCells:
    """The reference's per-cell radiation routines on independent cells
    (RADCELLS build, oracle/ref/harness.c): metric points, conserved
    variables and opacities of given primitives, u2p_rad and the implicit
    source solve solve_implicit_lab (rad.c:1225-1570)."""

    def __init__(self, libname="libkref_radcells.so"):
        self.L = _lib(os.path.join(REF_DIR, libname))
        self.L.kref_init()
        c = np.zeros(32)
        self.L.kref_rad_consts(_p(c))
        self.consts = c
        self.batch = int(c[24])

    def metric(self, r, th):
        g20, G20 = np.zeros(20), np.zeros(20)
        xx = np.array([0., r, th, 0.])
        self.L.kref_metric_at(_p(xx), _p(g20), _p(G20))
        return g20, G20

    def prepare(self, pp, g, G):
        """Sets the entropy slot of pp (in place); returns (uu, kappa_abs, kappa_es)."""
        n = pp.shape[0]
        uu, kap = np.zeros_like(pp), np.zeros((n, 2))
        self.L.kref_rad_prepare(n, _p(pp), _p(g), _p(G), _p(uu), _p(kap))
        return uu, kap[:, 0], kap[:, 1]

    def u2p(self, uu, pp, g, G):
        n = uu.shape[0]
        pp = pp.copy()
        st, co = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.L.kref_rad_u2p(n, _p(uu), _p(pp), _p(g), _p(G), _i(st), _i(co))
        return pp, st, co

    def u2p_full(self, uu, pp, g, G):
        """The reference's u2p (u2p.c:176, MHD then M1) per cell; returns
        (pp, status, corrected [n][3], fixups [n][2])."""
        n = uu.shape[0]
        pp = pp.copy()
        st = np.zeros(n, np.int32)
        co, fx = np.zeros((n, 3), np.int32), np.zeros((n, 2), np.int32)
        self.L.kref_u2p_full(n, _p(uu), _p(pp), _p(g), _p(G), _i(st), _i(co), _i(fx))
        return pp, st, co, fx

    # counter slot of the successful attempt -> (primitives, equation, frame)
    SLOTS = {0: ("RAD", "energy", "lab"), 13: ("RAD", "energy", "ff"), 2: ("MHD", "energy", "lab"),
             14: ("MHD", "energy", "ff"), 4: ("RAD", "entropy", "lab"), 6: ("MHD", "entropy", "lab")}

    def implicit(self, uu, pp, g, G, dt):
        """Returns (pp, uu, status, slot, iters); slot keys SLOTS (-1: all failed)."""
        n = uu.shape[0]
        po, uo = np.zeros_like(pp), np.zeros_like(uu)
        st, wh, it = (np.zeros(n, np.int32) for _ in range(3))
        for s in range(0, n, self.batch):
            m = min(self.batch, n - s)
            self.L.kref_rad_implicit(m, _p(uu[s:]), _p(pp[s:]), _p(g[s:]), _p(G[s:]), _p(dt[s:]), _p(po[s:]),
                                     _p(uo[s:]), _i(st[s:]), _i(wh[s:]), _i(it[s:]))
        return po, uo, st, wh, it

